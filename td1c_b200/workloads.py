"""Workload definitions (synthetic, seeded) for the orbital-equation RHS.

Each workload is a plain dict with the keys of td1c's input deck that the
hot path reads (clfedvr "grid:", clsph lmax1/lmax2/nlat, clbas "orbital:",
clormas nela/nelb/mtot/smul, clcontrol gauge, clfield1 pulse, clcrk dt).
Orbital tuples are (n, l, m, type) as in td1c's "orbital:" block with
type -1 = frozen core, 0 = dynamic core, 1 = active.

The two full-size workloads are the He TDHF and Ne TD-CASSCF atoms the
measurement is quoted on; the small ones are CPU-checkable variants with the
same code paths (frozen core, dynamic core, active space, both gauges).
"""

HE_TDHF = dict(
    name="he_tdhf_fedvr40x21_lmax23",
    znuc=2.0, rmin=0.0, rmax=80.0, ndvr=20, nfe=40, lmax1=23, lmax2=46, nlat=0,
    orbitals=[(1, 0, 0, 0)], nela=1, nelb=1, mtot=0, smul=1,
    igauge=1, icomp=1, rmask=60.0, mask_cos_order=8.0,
    fint=1.0e14, wlen=800.0, numcyc=3.0, cep=0.0, dt=0.005, seed=1,
)

NE_CAS = dict(
    name="ne_tdcasscf_fc1_cas8e9o_fedvr60x21_lmax47",
    znuc=10.0, rmin=0.0, rmax=120.0, ndvr=20, nfe=60, lmax1=47, lmax2=94, nlat=0,
    orbitals=[(1, 0, 0, -1),
              (2, 0, 0, 1), (2, 1, -1, 1), (2, 1, 0, 1), (2, 1, 1, 1),
              (3, 0, 0, 1), (3, 1, -1, 1), (3, 1, 0, 1), (3, 1, 1, 1), (3, 2, 0, 1)],
    nela=5, nelb=5, mtot=0, smul=1,
    igauge=1, icomp=1, rmask=96.0, mask_cos_order=4.0,
    fint=5.0e14, wlen=800.0, numcyc=4.0, cep=0.0, dt=0.004, seed=2,
)


def small(base, **kw):
    """A reduced-size copy of a workload (same orbital structure)."""
    wl = dict(base)
    wl.update(kw)
    wl["name"] = wl["name"] + "_small"
    return wl


# CPU-checkable cases covering every orbital class and both gauges
HE_SMALL = small(HE_TDHF, rmax=16.0, ndvr=8, nfe=8, lmax1=5, lmax2=10, rmask=12.0)
NE_SMALL = small(NE_CAS, rmax=16.0, ndvr=8, nfe=8, lmax1=5, lmax2=10, rmask=12.0)
MIXED_SMALL = dict(
    name="mixed_fc_dc_act_small",
    znuc=6.0, rmin=0.0, rmax=14.0, ndvr=7, nfe=8, lmax1=4, lmax2=8, nlat=0,
    orbitals=[(1, 0, 0, -1), (2, 0, 0, 0), (2, 1, -1, 1), (2, 1, 0, 1), (2, 1, 1, 1), (3, 0, 0, 1)],
    nela=3, nelb=3, mtot=0, smul=1,
    igauge=1, icomp=1, rmask=11.0, mask_cos_order=4.0,
    fint=1.0e14, wlen=800.0, numcyc=2.0, cep=30.0, dt=0.002, seed=3,
)
LENGTH_SMALL = dict(MIXED_SMALL, name="mixed_length_gauge_small", igauge=0, seed=4)
OPEN_SMALL = dict(MIXED_SMALL, name="open_shell_small", nela=4, nelb=3, smul=2, mtot=1, seed=5)

WORKLOADS = {w["name"]: w for w in [HE_TDHF, NE_CAS, HE_SMALL, NE_SMALL, MIXED_SMALL, LENGTH_SMALL, OPEN_SMALL]}
