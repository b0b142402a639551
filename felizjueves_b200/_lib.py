"""ctypes binding of libfjb.so (include/fjb.h).

The library is built in-tree (felizjueves_b200/build.py) and loaded from
felizjueves_b200/_lib/libfjb.so.  There is no fallback: a missing library
or a failing call raises.
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libfjb.so")

FJB_FP64 = 0
FJB_ROUTED = 1
FJB_FP64_SCATTER = 2  # FP64 without atomics: slot buffer + ordered per-element scatter

_ERRORS = {-1: ValueError, -2: RuntimeError, -3: RuntimeError, -4: ValueError,
           -5: TimeoutError, -6: ValueError}


class Basis_t(C.Structure):
    _fields_ = [("n_shells", C.c_int32), ("l", C.c_void_p), ("centre", C.c_void_p),
                ("prim0", C.c_void_p), ("nprim", C.c_void_p), ("exps", C.c_void_p),
                ("coefs", C.c_void_p)]


class PlanCounts_t(C.Structure):
    _fields_ = [(n, C.c_int64) for n in (
        "pairs", "pairs_deleted", "primitive_pairs", "primitive_pairs_pruned",
        "batches", "batch_pairs", "batch_pairs_screened", "launches",
        "kept_pairs", "kept_prims", "units", "quartets_launched")]


class PlanLists_t(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in (
        "batch_key", "batch_npairs", "pair_ab", "pair_mag", "prims",
        "pair_G", "pair_dmax", "pair_key", "prim_G",
        "launches", "screened", "deleted", "magnitudes", "eps", "g_max")]


class JLists_t(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("a", "b", "prim", "L", "G", "key", "ket_order", "L_off")]


_lib = None


def load():
    """The loaded library; raises if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libfjb.so is not built ({LIB_PATH}); run "
                           "`python -m felizjueves_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    L.fjb_last_error.restype = C.c_char_p
    L.fjb_last_error.argtypes = [vp]
    L.fjb_version.restype = C.c_char_p
    L.fjb_create.argtypes = [C.POINTER(vp), C.POINTER(Basis_t), C.c_int]
    L.fjb_destroy.argtypes = [vp]
    L.fjb_destroy.restype = None
    L.fjb_n_ao.argtypes = [vp]
    L.fjb_plan.argtypes = [vp, vp, dbl, C.c_int]
    L.fjb_plan_counts.argtypes = [vp, C.POINTER(PlanCounts_t)]
    L.fjb_plan_export.argtypes = [vp, C.POINTER(PlanLists_t)]
    L.fjb_screen_mask.argtypes = [vp, vp, vp, vp]
    L.fjb_fock_build.argtypes = [vp, vp, vp, vp, vp, C.c_int, dbl, vp]
    L.fjb_fock_build_host.argtypes = [vp, vp, vp, vp, vp, C.c_int, dbl]
    L.fjb_eri_blocks.argtypes = [vp, vp, C.c_int, vp, vp]
    L.fjb_eri_blocks_fp32.argtypes = [vp, vp, C.c_int, vp, vp]
    L.fjb_boys.argtypes = [C.c_int, vp, C.c_int, vp]
    L.fjb_last_build_stats.argtypes = [vp, C.POINTER(dbl), C.POINTER(C.c_int)]
    L.fjb_launch_stats.argtypes = [vp, vp, i64]
    L.fjb_class_stats.argtypes = [vp, vp, i64, C.POINTER(i64)]
    L.fjb_fma_probe.argtypes = [C.c_int, C.c_int, C.POINTER(dbl)]
    L.fjb_fock_build_noalloc.argtypes = [vp, vp, vp, vp, vp, vp]
    L.fjb_set_class_config.argtypes = [vp] + [C.c_int] * 6
    L.fjb_set_class_config32.argtypes = [vp] + [C.c_int] * 6
    L.fjb_set_rys.argtypes = [vp, C.c_int]
    L.fjb_set_route_check.argtypes = [vp, dbl, C.c_int]
    L.fjb_df_jk.argtypes = [vp, vp, i64, i64, vp, vp, vp, vp]
    L.fjb_hjk_plan.argtypes = [vp, vp, dbl, C.c_int, C.c_int]
    L.fjb_hjk_counts.argtypes = [vp, vp]
    L.fjb_hjk_export.argtypes = [vp, vp, vp, vp, vp]
    L.fjb_hjk_keys.argtypes = [vp, C.c_int, vp, vp]
    L.fjb_hjk_k.argtypes = [vp, vp, vp, vp]
    L.fjb_hjk_computed.argtypes = [vp, vp]
    L.fjb_df_eri3.argtypes = [vp, C.c_int, C.c_int, dbl, vp, C.POINTER(C.c_int32), vp]
    L.fjb_df_syrk.argtypes = [vp, vp, i64, i64, vp, vp]
    L.fjb_batch_create.argtypes = [C.POINTER(vp), vp, C.c_int]
    L.fjb_batch_set_densities.argtypes = [vp, vp, vp, vp, vp]
    L.fjb_batch_build.argtypes = [vp, C.c_int, dbl, vp]
    L.fjb_batch_stats.argtypes = [vp, C.POINTER(dbl), C.POINTER(i64), C.POINTER(i64)]
    L.fjb_batch_last_error.restype = C.c_char_p
    L.fjb_batch_last_error.argtypes = [vp]
    L.fjb_batch_destroy.argtypes = [vp]
    L.fjb_batch_destroy.restype = None
    L.fjb_route_check_result.argtypes = [vp, C.POINTER(dbl), C.POINTER(C.c_int)]
    L.fjb_fock_build_graph.argtypes = [vp, vp, vp, vp, vp, C.c_int, dbl, vp]
    L.fjb_create_df.argtypes = [C.POINTER(vp), C.POINTER(Basis_t), C.POINTER(Basis_t), C.c_int]
    L.fjb_df_blocks.argtypes = [vp, C.c_int, vp, C.c_int, vp, vp]
    L.fjb_mlp_n_params.argtypes = []
    L.fjb_router_set.argtypes = [vp, vp, C.c_float]
    L.fjb_router_reach.argtypes = [vp, dbl]
    L.fjb_router_classes.argtypes = [vp, C.c_int]
    L.fjb_router_features.argtypes = [vp, vp, vp, C.c_int, vp, vp]
    L.fjb_mlp_forward.argtypes = [vp, vp, C.c_int, vp, vp]
    L.fjb_mlp_forward_tc.argtypes = [vp, vp, C.c_int, vp, vp]
    L.fjb_plan_units.argtypes = [vp, vp, i64, C.POINTER(i64)]
    L.fjb_mlp_gradient.argtypes = [vp, vp, vp, C.c_int, vp, vp, vp, vp]
    L.fjb_mlp_adam.argtypes = [vp, vp, vp, vp, C.c_float, C.c_int, vp]
    L.fjb_route_stats.argtypes = [vp, C.POINTER(i64), C.POINTER(i64)]
    L.fjb_coulomb.argtypes = [vp, vp, vp, dbl, vp]
    L.fjb_coulomb_mixed.argtypes = [vp, vp, vp, dbl, dbl, vp]
    L.fjb_j_last_launches.argtypes = [vp]
    L.fjb_j_plan_lists.argtypes = [vp, vp, C.POINTER(JLists_t), C.POINTER(i64)]
    L.fjb_scatter_map.argtypes = [vp, C.c_int, vp, vp, vp, C.POINTER(i64), C.POINTER(i64)]
    L.fjb_one_electron.argtypes = [vp, vp, vp, C.c_int, vp, vp, vp, vp, vp]
    _lib = L
    return L


EXPORTS = ("fjb_last_error", "fjb_version", "fjb_create", "fjb_destroy", "fjb_n_ao",
           "fjb_plan", "fjb_plan_counts", "fjb_plan_export", "fjb_screen_mask",
           "fjb_fock_build", "fjb_fock_build_host", "fjb_eri_blocks", "fjb_eri_blocks_fp32", "fjb_boys",
           "fjb_last_build_stats", "fjb_launch_stats", "fjb_class_stats",
           "fjb_fma_probe", "fjb_fock_build_noalloc", "fjb_set_class_config", "fjb_set_class_config32",
           "fjb_set_rys", "fjb_set_route_check", "fjb_route_check_result", "fjb_df_jk", "fjb_df_eri3", "fjb_df_syrk",
           "fjb_hjk_plan", "fjb_hjk_counts", "fjb_hjk_export", "fjb_hjk_keys", "fjb_hjk_k", "fjb_hjk_computed",
           "fjb_batch_create", "fjb_batch_set_densities", "fjb_batch_build", "fjb_batch_stats",
           "fjb_batch_last_error", "fjb_batch_destroy",
           "fjb_fock_build_graph", "fjb_create_df", "fjb_df_blocks", "fjb_mlp_n_params",
           "fjb_router_set", "fjb_router_reach", "fjb_router_classes", "fjb_router_features", "fjb_mlp_forward", "fjb_mlp_forward_tc",
           "fjb_mlp_gradient", "fjb_plan_units",
           "fjb_mlp_adam", "fjb_route_stats", "fjb_coulomb", "fjb_coulomb_mixed", "fjb_j_last_launches",
           "fjb_j_plan_lists", "fjb_scatter_map", "fjb_one_electron")


class LaunchStat_t(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("la", "lb", "lc", "ld", "kab", "kcd")] + \
               [("launched", C.c_int64), ("computed", C.c_int64)]


class ClassStat_t(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("la", "lb", "lc", "ld")] + \
               [("ms", C.c_double), ("units", C.c_int64), ("engine", C.c_int32), ("pad", C.c_int32)]


def check(rc: int, handle=None) -> None:
    if rc == 0:
        return
    msg = load().fjb_last_error(handle).decode(errors="replace")
    raise _ERRORS.get(rc, RuntimeError)(f"fjb error {rc}: {msg}")
