"""Algorithmic work per RHS phase (FLOPs and compulsory HBM bytes).

Counts follow the loops of the reference routines with the m-selection and
l >= |m| bounds applied (only work the reference performs is counted):
  orbin      sph2ang1 over dynamic orbitals           bas_sph2ang1.F90:88-156
  rho_gemm   pair products + theta->l                 hprod_mkrho2.F90, bas_ang2sph2.F90:330-482
  poisson    per (pair, l): element shares, bridge solve, interior products
             (static condensation of the same linear system)  hprod_mkv2mf.F90:118-182
  w_gemm     l->theta                                 bas_sph2ang2.F90:334-463
  mfprod     core J/K + active J/K + 2-RDM contraction hprod_mfprod2.F90
  gorb_gemm  theta->l of g and v2                     bas_ang2sph1.F90:88-158
  orbdots    orbital matrix elements                  hprod_mkint1_sph.F90, hprod_htot_mkxmat.F90
  int2e      (ij|kl) over Nr (lmax2+1)                hprod_mkint2_sph.F90:2-100
  onebody    banded tmat/pmat stencils + laser        hprod_tprod/zprod/pzprod.F90
  dtorb      orbital time derivative                  hprod_htot_dtorb.F90
Bytes are the compulsory HBM traffic of each phase: every array it must read
once and write once (tables that stay L2-resident are not counted).
"""


def rhs_work(wl, dims):
    orbs = wl["orbitals"]
    nfun = len(orbs)
    m = [o[2] for o in orbs]
    t = [o[3] for o in orbs]
    nfc = sum(1 for x in t if x == -1)
    ncore = sum(1 for x in t if x <= 0)
    nact = nfun - ncore
    Nr = dims["nrad"] - 1
    L1, L2 = wl["lmax1"] + 1, wl["lmax2"] + 1
    nlat = dims["nlat"]
    nd = wl["ndvr"]
    nbas, nbas2, ngrid = Nr * L1, Nr * L2, Nr * nlat
    C = 16  # bytes per complex128
    dyn = list(range(nfc, nfun))
    pairs = [(a, b) for b in dyn for a in range(b, nfun)] + [(a, b) for b in range(nfc) for a in dyn]
    npair = len(pairs)
    w = {}
    # orbin
    f_orbin = sum((L1 - abs(m[f])) * nlat * 2 * Nr * 2 for f in dyn)
    w["orbin"] = (f_orbin, C * len(dyn) * (nbas + ngrid))
    # pair density + theta->l
    f_rho = sum((L2 - abs(m[b] - m[a])) * nlat * 2 * Nr * 2 + 6 * nlat * Nr for a, b in pairs)
    w["rho_gemm"] = (f_rho, C * (nfun * ngrid + npair * nbas2))
    # Poisson by static condensation, per complex (pair, l) system: three share rows over
    # the nd owned points of each element, the interior products (ni x ni, real matrix on
    # complex data) with their finalisation, and the tridiagonal bridge solve.  Bytes: rho2
    # read by the share and the element passes, v2sph written once, the per-(l, element)
    # records read once.
    nfe, ni = (Nr + 1) // nd, nd - 1
    nsys = sum(L2 - abs(m[b] - m[a]) for a, b in pairs)
    f_sys = nfe * (3 * nd * 4 + ni * ni * 4 + ni * 8 + 8) + (nfe - 1) * 16
    rec = 8 * L2 * nfe * ((ni * ni + 3 * ni + 3) // 2 * 2 + (3 * nd + 1) // 2 * 2)
    w["poisson"] = (nsys * f_sys, C * 3 * npair * nbas2 + rec)
    # l->theta
    f_w = sum(nlat * (L2 - abs(m[b] - m[a])) * 2 * Nr * 2 for a, b in pairs)
    w["w_gemm"] = (f_w, C * npair * (nbas2 + ngrid))
    # mfprod: act2 entries + fc/dc terms + twfn + rden
    nent = 0
    for ia in range(nact):
        for ja in range(ia + 1):
            for ka in range(nact):
                for la in range(nact):
                    i, j, k, l = ncore + ia, ncore + ja, ncore + ka, ncore + la
                    if m[i] + m[k] == m[j] + m[l]:
                        nent += 1
    npair_act = nact * (nact + 1) // 2
    nsame = sum(1 for a in range(ncore, nfun) for b in range(ncore, nfun) if m[a] == m[b])
    f_mf = ngrid * (8 * nent + 8 * nfc * len(dyn) + 16 * npair_act + 8 * nsame)
    w["mfprod"] = (f_mf, C * ngrid * (npair + nfun + 2 * len(dyn)))
    # theta->l of g, v2
    f_g = 2 * sum((L1 - abs(m[f])) * nlat * 2 * Nr * 2 for f in dyn)
    w["gorb_gemm"] = (f_g, C * 2 * len(dyn) * (ngrid + nbas))
    # orbital matrix elements
    nsame_all = sum(1 for a in range(nfun) for b in dyn if m[a] == m[b])
    w["orbdots"] = (8 * nbas * 2 * nsame_all, C * 5 * nfun * nbas)
    # int2e
    nq = 0
    for ia in range(nact):
        for ja in range(ia + 1):
            for ka in range(nact):
                for la in range(nact):
                    i, j, k, l = ncore + ia, ncore + ja, ncore + ka, ncore + la
                    if m[i] + m[k] == m[j] + m[l]:
                        nq += 1
    w["int2e"] = (8 * nq * nbas2, C * 2 * npair_act * nbas2)
    # one-body stencils
    nchan = sum(L1 - abs(m[f]) for f in range(nfun))
    f_ob = nchan * Nr * (2 * nd + 1) * 4 * (2 if wl["igauge"] == 1 else 1) + nchan * Nr * 16
    w["onebody"] = (f_ob, C * 3 * nfun * nbas)
    # dtorb
    f_dt = len(dyn) * nbas * (6 + 8 + 8 * sum(1 for a in range(nfun) if True))
    w["dtorb"] = (f_dt, C * (6 * nfun * nbas))
    return w
