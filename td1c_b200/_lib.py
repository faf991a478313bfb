"""Build and load libtd1c_b200.so (the sm_100a CUDA library with the C-ABI).

The library is built in-tree by nvcc for sm_100a.  Loading never falls back
to anything else: if the shared library is missing or fails to load, the
error propagates.
"""
import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
LIB_PATH = os.path.join(LIB_DIR, "libtd1c_b200.so")
SOURCES = ["hprod.cu", "legendre_gemm.cu", "onebody.cu", "poisson.cu", "mfprod.cu", "reductions.cu", "ci.cu",
           "int2e_static.cu", "int2e_dmma.cu", "observables.cu", "h1prop.cu", "poisson_cond.cu",
           "legendre_tf32.cu", "legendre_tc.cu", "int2e_tc.cu", "mlp.cu",
           "predictor.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]

_lib = None


def build(verbose=False):
    """Compile every CUDA source into td1c_b200/_lib/libtd1c_b200.so (one object per
    source, compiled in parallel, then linked)."""
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(LIB_DIR, exist_ok=True)
    obj_dir = os.path.join(LIB_DIR, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    objs, cmds = [], []
    for s in SOURCES:
        o = os.path.join(obj_dir, s.replace(".cu", ".o"))
        objs.append(o)
        cmds.append([NVCC] + compile_flags + ["-c", "-o", o, os.path.join(CSRC, s)])
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for cmd, r in zip(cmds, ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds)):
            if verbose:
                print(" ".join(cmd))
            if r.returncode != 0:
                raise RuntimeError("nvcc failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    link = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB_PATH] + objs
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    return LIB_PATH


def _newer_sources():
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    for f in os.listdir(CSRC):
        if os.path.getmtime(os.path.join(CSRC, f)) > t:
            return True
    return False


def load():
    """Load the CUDA library (building it first if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = ctypes.CDLL(LIB_PATH)
    c_int, c_double, c_long, vp = ctypes.c_int, ctypes.c_double, ctypes.c_long, ctypes.c_void_p
    dp, ip, up = ctypes.POINTER(c_double), ctypes.POINTER(c_int), ctypes.POINTER(ctypes.c_uint)
    lib.td1c_gpu_bind_rad.argtypes = [c_int, c_int, c_int, dp, dp, dp, dp, dp, c_double, dp]
    lib.td1c_gpu_bind_sph.argtypes = [c_int, c_int, c_int, c_int, c_int, dp, dp, dp, dp, dp, dp]
    lib.td1c_gpu_bind_bas.argtypes = [c_double, c_int, c_int, c_int, ip, ip, ip, c_int, c_int]
    lib.td1c_gpu_bind_control.argtypes = [c_int, c_int]
    lib.hprod_bind_.argtypes = [dp, dp, dp, dp, dp, dp, dp, dp, ctypes.POINTER(ctypes.c_bool), dp]
    lib.hprod_init_.argtypes = []
    lib.hprod_set_wfn0_.argtypes = [dp, dp, ctypes.c_char_p, c_int]
    lib.hprod_htot_.argtypes = [dp, dp, dp, dp, dp, dp]
    lib.hprod_final_.argtypes = []
    lib.td1c_gpu_last_status.restype = c_int
    lib.td1c_gpu_dims.argtypes = [ip]
    lib.td1c_gpu_ci_tables.argtypes = [up, up, ip, ip, ip]
    lib.td1c_gpu_energies.argtypes = [dp]
    lib.td1c_gpu_htot_dev.argtypes = [c_double, dp, vp, vp, vp, vp]
    lib.td1c_gpu_debug_get.restype = c_long
    lib.td1c_gpu_debug_get.argtypes = [ctypes.c_char_p, dp, c_long]
    lib.td1c_gpu_rk4.argtypes = [vp, vp, c_double, c_double, c_int, c_double, c_double, c_double, c_double, c_int]
    lib.td1c_gpu_sync.restype = c_int
    lib.td1c_gpu_launch_count.restype = c_long
    lib.td1c_gpu_stream.restype = vp
    lib.td1c_gpu_rk4_reset.argtypes = [vp, vp]
    lib.td1c_gpu_profile.restype = c_int
    lib.td1c_gpu_profile.argtypes = [c_int, c_double, dp, vp, vp, vp, vp, dp, ctypes.c_char_p, c_int]
    lib.td1c_gpu_orth.restype = c_int
    lib.td1c_gpu_orth.argtypes = [vp, vp]
    lib.td1c_gpu_relax.restype = c_int
    lib.td1c_gpu_relax.argtypes = [vp, vp, c_double, c_int, dp]
    lib.td1c_gpu_dipole.restype = c_int
    lib.td1c_gpu_dipole.argtypes = [vp, vp, dp]
    lib.td1c_gpu_dipole3.restype = c_int
    lib.td1c_gpu_dipole3.argtypes = [vp, vp, dp, dp]
    lib.td1c_gpu_set_mixed.restype = c_int
    lib.td1c_gpu_set_mixed.argtypes = [c_int]
    lib.td1c_gpu_mixed_selftest.restype = c_int
    lib.td1c_gpu_mixed_selftest.argtypes = [vp, vp, dp, dp]
    lib.td1c_gpu_mixed_int2e_selftest.restype = c_int
    lib.td1c_gpu_mixed_int2e_selftest.argtypes = [vp, vp, dp, dp]
    lib.hprod_dipole_.restype = None
    lib.hprod_dipole_.argtypes = [dp, dp, dp, dp, dp, dp]
    lib.td1c_gpu_int2e_static.restype = c_int
    lib.td1c_gpu_int2e_static.argtypes = [c_int, ip, c_long, vp, vp, vp, vp]
    lib.td1c_gpu_bind_split.restype = c_int
    lib.td1c_gpu_bind_split.argtypes = [c_int]
    lib.td1c_gpu_h1itr.restype = c_int
    lib.td1c_gpu_h1itr.argtypes = [vp, dp, c_double, c_int, c_double, ip]
    lib.td1c_gpu_dpade.restype = c_int
    lib.td1c_gpu_dpade.argtypes = [vp, dp, c_double, c_double, c_double, c_int, c_double, ip]
    for name in ("td1c_gpu_split2", "td1c_gpu_etdrk2", "td1c_gpu_etdrk4"):
        getattr(lib, name).restype = c_int
        getattr(lib, name).argtypes = [vp, vp, c_double, c_double, c_int, c_double, c_double, c_double, c_double,
                                       c_int, c_double, c_int]
    lib.td1c_gpu_relax_etdrk2.restype = c_int
    lib.td1c_gpu_relax_etdrk2.argtypes = [vp, vp, c_double, c_int, c_int, c_double, dp]
    lib.h1itr_gen_cninv_.argtypes = [ip, dp, ip, dp]
    lib.h1itr_prop_.argtypes = [ip, ip, ip, ip, dp, dp, ip, dp, ip, dp, dp]
    lib.dpade_gen_.argtypes = [ip, dp, dp, dp, ip]
    lib.dpade_prod_.argtypes = [ip, ip, ip, ip, dp, dp, dp, ip, dp, ip, dp, dp]
    lib.td1c_gpu_debug_ptr.restype = vp
    lib.td1c_gpu_debug_ptr.argtypes = [ctypes.c_char_p]
    lib.td1c_gpu_debug_xfer.restype = c_long
    lib.td1c_gpu_debug_xfer.argtypes = [ctypes.c_char_p, vp, c_int]
    lib.td1c_gpu_set_mf_external.restype = c_int
    lib.td1c_gpu_set_mf_external.argtypes = [c_int]
    fpp = ctypes.POINTER(ctypes.c_void_p)
    lib.td1c_mlp_forward.restype = c_int
    lib.td1c_mlp_forward.argtypes = [c_int, ip, fpp, fpp, vp, c_int, vp, vp]
    lib.td1c_mlp_backward.restype = c_int
    lib.td1c_mlp_backward.argtypes = [c_int, ip, fpp, vp, c_int, vp, vp, fpp, fpp, vp, vp]
    lib.td1c_mlp_adam.restype = c_int
    lib.td1c_mlp_adam.argtypes = [c_long, vp, vp, vp, vp, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                  c_int, vp]
    lib.td1c_mlp_pack_size.restype = c_long
    lib.td1c_mlp_pack_size.argtypes = [c_int, ip]
    lib.td1c_mlp_infer_bf16.restype = c_int
    lib.td1c_mlp_infer_bf16.argtypes = [c_int, ip, fpp, fpp, vp, c_int, vp, c_int, vp, vp, vp]
    lib.td1c_gpu_set_learned.restype = c_int
    lib.td1c_gpu_set_learned.argtypes = [c_int, ip, fpp, fpp, vp, c_int, c_double]
    lib.td1c_gpu_set_learned_policy.restype = c_int
    lib.td1c_gpu_set_learned_policy.argtypes = [c_int]
    lib.td1c_gpu_split2_learned.restype = c_int
    lib.td1c_gpu_split2_learned.argtypes = [vp, vp, c_double, c_double, c_int, c_double, c_double, c_double, c_double, c_int,
                                            c_double, dp]
    lib.td1c_gpu_learned_record.restype = c_int
    lib.td1c_gpu_learned_record.argtypes = [vp, vp, c_double, c_double, c_int, c_double, c_double, c_double, c_double, c_int,
                                            c_double, vp]
    lib.td1c_gpu_learned_dims.restype = c_int
    lib.td1c_gpu_learned_dims.argtypes = [ip]
    lib.td1c_gpu_learned_pair_kind.restype = c_int
    lib.td1c_gpu_learned_pair_kind.argtypes = [ip]
    lib.td1c_lp_features.restype = c_int
    lib.td1c_lp_features.argtypes = [c_int, vp, vp, c_int, c_int, vp, vp, vp]
    lib.td1c_lp_loss.restype = c_int
    lib.td1c_lp_loss.argtypes = [c_int, vp, vp, vp, vp, vp, c_int, vp]
    for name in ("td1c_gpu_ctx_create", "td1c_gpu_ctx_current"):
        getattr(lib, name).restype = c_int
        getattr(lib, name).argtypes = []
    for name in ("td1c_gpu_ctx_select", "td1c_gpu_ctx_destroy"):
        getattr(lib, name).restype = c_int
        getattr(lib, name).argtypes = [c_int]
    lib.td1c_gpu_set_tuning.restype = c_int
    lib.td1c_gpu_set_tuning.argtypes = [c_int, c_int, c_int]
    lib.td1c_gpu_get_tuning.restype = c_int
    lib.td1c_gpu_get_tuning.argtypes = [ip]
    lib.td1c_gpu_ensemble_split2.restype = c_int
    lib.td1c_gpu_ensemble_split2.argtypes = [c_int, ip, fpp, fpp, dp, dp, c_int, dp, dp, dp, dp, c_int, c_double, dp]
    lib.td1c_gpu_bind_ormas.restype = c_int
    lib.td1c_gpu_bind_ormas.argtypes = [c_int]
    lib.td1c_gpu_wait_selftest.restype = c_int
    lib.td1c_gpu_wait_selftest.argtypes = []
    lib.td1c_gpu_pulse_lfield.restype = c_int
    lib.td1c_gpu_pulse_lfield.argtypes = [c_double, c_double, c_double, c_double, c_double, dp]
    _lib = lib
    return lib


EXPORTED = [
    "td1c_gpu_bind_rad", "td1c_gpu_bind_sph", "td1c_gpu_bind_bas", "td1c_gpu_bind_control",
    "hprod_bind_", "hprod_init_", "hprod_set_wfn0_", "hprod_htot_", "hprod_final_",
    "td1c_gpu_last_status", "td1c_gpu_dims", "td1c_gpu_ci_tables", "td1c_gpu_energies",
    "td1c_gpu_htot_dev", "td1c_gpu_debug_get", "td1c_gpu_rk4", "td1c_gpu_sync", "td1c_gpu_launch_count",
    "td1c_gpu_stream", "td1c_gpu_profile", "td1c_gpu_rk4_reset", "td1c_gpu_int2e_static", "td1c_gpu_dipole",
    "td1c_gpu_dipole3", "hprod_dipole_", "td1c_gpu_set_mixed", "td1c_gpu_mixed_selftest", "td1c_gpu_mixed_int2e_selftest",
    "td1c_gpu_orth", "td1c_gpu_relax", "td1c_gpu_bind_split", "td1c_gpu_h1itr", "td1c_gpu_dpade",
    "td1c_gpu_split2", "td1c_gpu_etdrk2", "td1c_gpu_etdrk4", "td1c_gpu_relax_etdrk2",
    "h1itr_gen_cninv_", "h1itr_prop_", "dpade_gen_", "dpade_prod_",
    "td1c_gpu_debug_ptr", "td1c_gpu_debug_xfer", "td1c_gpu_set_mf_external", "td1c_gpu_pulse_lfield",
    "td1c_gpu_bind_ormas", "td1c_gpu_wait_selftest",
    "td1c_mlp_forward", "td1c_mlp_backward", "td1c_mlp_adam", "td1c_mlp_pack_size", "td1c_mlp_infer_bf16",
    "td1c_gpu_set_learned", "td1c_gpu_set_learned_policy", "td1c_gpu_split2_learned", "td1c_gpu_learned_record", "td1c_gpu_learned_dims",
    "td1c_gpu_learned_pair_kind", "td1c_lp_features", "td1c_lp_loss",
    "td1c_gpu_ctx_create", "td1c_gpu_ctx_select", "td1c_gpu_ctx_current", "td1c_gpu_ctx_destroy",
    "td1c_gpu_set_tuning", "td1c_gpu_get_tuning", "td1c_gpu_ensemble_split2",
]
