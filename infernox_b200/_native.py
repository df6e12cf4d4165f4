"""ctypes binding of libcmscan_gpu.so (include/cmscan_gpu.h).

The library is built in-tree (infernox_b200/_lib) by infernox_b200.build; it
is loaded from there and nowhere else.  A missing library is an error: there
is no CPU fallback for the scanner.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libcmscan_gpu.so")

CMGPU_OK = 0
CMGPU_EINVAL = -1
CMGPU_ENOMEM = -2
CMGPU_EDEVICE = -3
CMGPU_EOVERFLOW = -4
CMGPU_ERANGE = -5
CMGPU_ETIMEOUT = -6
CMGPU_ENOSPACE = -7
CYK_F32, INSIDE_I32, INSIDE_F32 = 0, 1, 2
NOQDB, QDB1, QDB2 = 0, 1, 2
KERNEL_AUTO, KERNEL_LEVEL, KERNEL_SWEEP = 0, 1, 2

P = C.POINTER


class CmParams(C.Structure):
    _fields_ = [
        ("M", C.c_int32), ("nodes", C.c_int32), ("clen", C.c_int32),
        ("sttype", P(C.c_int8)), ("stid", P(C.c_int8)), ("ndtype", P(C.c_int8)),
        ("ndidx", P(C.c_int32)), ("cfirst", P(C.c_int32)), ("cnum", P(C.c_int32)),
        ("plast", P(C.c_int32)), ("pnum", P(C.c_int32)), ("nodemap", P(C.c_int32)),
        ("t", P(C.c_float)), ("e", P(C.c_float)),
        ("null", C.c_float * 4),
        ("el_selfsc", C.c_float), ("pbegin", C.c_float), ("pend", C.c_float),
        ("n3_omega", C.c_float),
    ]


class TrPrep(C.Structure):
    _fields_ = [
        ("lmesc", P(C.c_float)), ("rmesc", P(C.c_float)),
        ("ilmesc", P(C.c_int32)), ("irmesc", P(C.c_int32)),
        ("pty", P(C.c_float)), ("ipty", P(C.c_int32)),
        ("lpos", P(C.c_int32)), ("rpos", P(C.c_int32)),
    ]


class Cm(C.Structure):
    _fields_ = [
        ("M", C.c_int32), ("W", C.c_int32), ("flags", C.c_uint32),
        ("sttype", P(C.c_int8)), ("stid", P(C.c_int8)),
        ("cfirst", P(C.c_int32)), ("cnum", P(C.c_int32)),
        ("tsc", P(C.c_float)), ("oesc", P(C.c_float)), ("endsc", P(C.c_float)),
        ("beginsc", P(C.c_float)), ("el_selfsc", C.c_float),
        ("itsc", P(C.c_int32)), ("ioesc", P(C.c_int32)), ("iendsc", P(C.c_int32)),
        ("ibeginsc", P(C.c_int32)), ("iel_selfsc", C.c_int32),
        ("dmin1", P(C.c_int32)), ("dmax1", P(C.c_int32)),
        ("dmin2", P(C.c_int32)), ("dmax2", P(C.c_int32)),
        ("null", C.c_float * 4), ("n3_omega", C.c_float),
    ]


class CmScores(C.Structure):
    _fields_ = [
        ("tsc", P(C.c_float)), ("oesc", P(C.c_float)), ("endsc", P(C.c_float)),
        ("beginsc", P(C.c_float)),
        ("itsc", P(C.c_int32)), ("ioesc", P(C.c_int32)), ("iendsc", P(C.c_int32)),
        ("ibeginsc", P(C.c_int32)),
        ("dmin1", P(C.c_int32)), ("dmax1", P(C.c_int32)),
        ("dmin2", P(C.c_int32)), ("dmax2", P(C.c_int32)),
        ("t_local", P(C.c_float)),
        ("el_selfsc", C.c_float), ("iel_selfsc", C.c_int32), ("W", C.c_int32),
        ("flags", C.c_uint32),
    ]


class P7Profile(C.Structure):
    _fields_ = [("M", C.c_int32), ("mat", P(C.c_float)), ("trans", P(C.c_float))]


class Cp9(C.Structure):
    """cmgpu_cp9: the CP9 HMM of a CM (caller-allocated arrays)."""
    _fields_ = [("M", C.c_int32), ("mat", P(C.c_float)), ("ins", P(C.c_float)), ("t", P(C.c_float)),
                ("begin", P(C.c_float)), ("end", P(C.c_float)), ("msc", P(C.c_int32)), ("isc", P(C.c_int32)),
                ("otsc", P(C.c_int32)), ("has_el", P(C.c_uint8)), ("hns2cs", P(C.c_int32)),
                ("el_pairs", P(C.c_int32)), ("n_el", C.c_int32), ("el_self", C.c_float), ("el_selfsc", C.c_int32)]


class F3Config(C.Structure):
    """cmgpu_f3_config: stages and thresholds of one f3_filter_sequence pass."""
    _fields_ = [("f1", C.c_double), ("f1b", C.c_double), ("f2", C.c_double), ("f2b", C.c_double),
                ("f3", C.c_double), ("f3b", C.c_double), ("cmw", C.c_int64), ("maxw", C.c_int64),
                ("do_msv", C.c_int32), ("do_msvbias", C.c_int32), ("do_vit", C.c_int32),
                ("do_vitbias", C.c_int32), ("do_fwd", C.c_int32), ("do_fwdbias", C.c_int32),
                ("lmmu", C.c_double), ("lmlambda", C.c_double), ("lvmu", C.c_double), ("lvlambda", C.c_double)]


F3_ACCT_FIELDS = ("n_past_msv", "pos_past_msv", "n_past_msvbias", "pos_past_msvbias", "n_past_vit", "pos_past_vit",
                  "n_past_vitbias", "pos_past_vitbias", "n_past_fwd", "pos_past_fwd", "n_past_fwdbias",
                  "pos_past_fwdbias")


class F3Acct(C.Structure):
    _fields_ = [(k, C.c_int64) for k in F3_ACCT_FIELDS]


class Hit(C.Structure):
    _fields_ = [("i", C.c_int32), ("j", C.c_int32), ("score", C.c_float), ("bias", C.c_float)]


HIT_DTYPE = np.dtype([("i", np.int32), ("j", np.int32), ("score", np.float32), ("bias", np.float32)])
BATCH_HIT_DTYPE = np.dtype([("win", np.int32), ("i", np.int32), ("j", np.int32),
                            ("score", np.float32), ("bias", np.float32)])
ENV_DTYPE = np.dtype([("start", np.int32), ("end", np.int32)])
WINDOW_DTYPE = np.dtype([("dsq_offset", np.int64), ("i0", np.int32), ("j0", np.int32)])


class HbBands(C.Structure):
    _fields_ = [("jmin", P(C.c_int32)), ("jmax", P(C.c_int32)), ("hd_off", P(C.c_int32)),
                ("hdmin", P(C.c_int32)), ("hdmax", P(C.c_int32))]


class HbTask(C.Structure):
    _fields_ = [("dsq_offset", C.c_int64), ("i0", C.c_int32), ("j0", C.c_int32), ("env_cutoff", C.c_float),
                ("cutoff", C.c_float), ("bands", HbBands)]


class TrTables(C.Structure):
    _fields_ = [("lmesc", P(C.c_float)), ("rmesc", P(C.c_float)), ("pty", P(C.c_float)),
                ("lpos", P(C.c_int32)), ("rpos", P(C.c_int32)), ("clen", C.c_int32), ("local", C.c_int32),
                ("ilmesc", P(C.c_int32)), ("irmesc", P(C.c_int32)), ("ipty", P(C.c_int32))]


class TrqResult(C.Structure):
    _fields_ = [("vsc_root", C.c_float), ("vmode", C.c_int32), ("bsc_full", C.c_float), ("nhits", C.c_int32),
                ("hit_first", C.c_int64)]


class TrTask(C.Structure):
    _fields_ = [("dsq_offset", C.c_int64), ("i0", C.c_int32), ("j0", C.c_int32), ("env_cutoff", C.c_float),
                ("cutoff", C.c_float), ("bands", HbBands), ("jvalid", P(C.c_uint8)), ("lvalid", P(C.c_uint8)),
                ("rvalid", P(C.c_uint8)), ("tvalid", P(C.c_uint8))]


class TrResult(C.Structure):
    _fields_ = [("vsc_root", C.c_float), ("vmode", C.c_int32), ("envi", C.c_int64), ("envj", C.c_int64),
                ("hit_first", C.c_int64), ("nhits", C.c_int32), ("pad", C.c_int32)]


TR_HIT_DTYPE = np.dtype([("i", np.int32), ("j", np.int32), ("score", np.float32), ("bias", np.float32),
                         ("mode", np.int32), ("root", np.int32)])


class HbResult(C.Structure):
    _fields_ = [("vsc_root", C.c_float), ("nhits", C.c_int32), ("envi", C.c_int64), ("envj", C.c_int64),
                ("hit_first", C.c_int64)]


class Stats(C.Structure):
    _fields_ = [
        ("cells", C.c_double), ("terms", C.c_double), ("residues", C.c_double),
        ("work_items", C.c_int64), ("candidates", C.c_int64),
        ("kernel_ms", C.c_float), ("kernel_launches", C.c_int32),
        ("deck_in_smem", C.c_int32), ("ctas", C.c_int32), ("lanes", C.c_int32),
        ("kernel", C.c_int32),
    ]


class CalibrateConfig(C.Structure):
    _fields_ = [("seed", C.c_uint32), ("l_mb", C.c_double), ("beta", C.c_double), ("nonbanded", C.c_int32),
                ("gtailn", C.c_int32), ("ltailn", C.c_int32), ("tailp", C.c_float), ("do_null3", C.c_int32)]


class ExpParams(C.Structure):
    _fields_ = [("lambda_", C.c_double), ("mu", C.c_double), ("dbsize", C.c_double), ("mu_orig", C.c_double),
                ("tailp", C.c_double), ("nrandhits", C.c_int32)]


class CalibrateResult(C.Structure):
    _fields_ = [("exp", ExpParams * 4), ("nhits", C.c_int32 * 4), ("dbsize", C.c_double), ("cells", C.c_double),
                ("terms", C.c_double), ("kernel_ms", C.c_float), ("launches", C.c_int32)]


def ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(P(ctype))


_lib = None


class CmgpuError(RuntimeError):
    def __init__(self, rc: int, msg: str):
        super().__init__(f"cmgpu error {rc}: {msg}")
        self.rc = rc


def lib() -> C.CDLL:
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m infernox_b200.build` first")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.cmgpu_last_error.restype = C.c_char_p
    L.cmgpu_version.restype = C.c_char_p
    L.cmgpu_prep_configure.argtypes = [P(CmParams), C.c_int, C.c_int32, C.c_double, C.c_double,
                                       C.c_double, P(CmScores)]
    L.cmgpu_prep_truncated.argtypes = [P(CmParams), C.c_int, P(TrPrep)]
    L.cmgpu_ilogsum_table.argtypes = [P(C.c_int32), C.c_int32]
    L.cmgpu_flogsum_table.argtypes = [P(C.c_float), C.c_int32]
    L.cmgpu_model_upload.argtypes = [P(Cm), C.c_int, P(vp)]
    L.cmgpu_model_free.argtypes = [vp]
    L.cmgpu_model_free.restype = None
    L.cmgpu_workspace_create.argtypes = [C.c_int, vp, P(vp)]
    L.cmgpu_workspace_free.argtypes = [vp]
    L.cmgpu_workspace_free.restype = None
    L.cmgpu_workspace_stats.argtypes = [vp, P(Stats)]
    L.cmgpu_workspace_set_shape.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int]
    L.cmgpu_workspace_set_kernel.argtypes = [vp, C.c_int]
    L.cmgpu_qdb_scan.argtypes = [vp, vp, C.c_int, C.c_int, P(C.c_uint8), C.c_int32, C.c_int32,
                                 C.c_int32, C.c_float, C.c_int, vp, C.c_int32, P(C.c_int32)]
    L.cmgpu_qdb_scan_noalloc.argtypes = [vp, vp, C.c_int, C.c_int, P(C.c_uint8), C.c_int32, C.c_int32,
                                         C.c_int32, C.c_float, C.c_int, vp, C.c_int32, P(C.c_int32)]
    L.cmgpu_qdb_scan_cells.argtypes = [vp, vp, C.c_int, C.c_int, P(C.c_uint8), C.c_int32, C.c_int32,
                                       C.c_int32, C.c_float, vp, vp, vp, C.c_int32, P(C.c_int32)]
    L.cmgpu_cyk_seq_filter.argtypes = [vp, vp, P(C.c_uint8), C.c_int32, C.c_float, C.c_int, vp,
                                       C.c_int32, P(C.c_int32)]
    L.cmgpu_final_stage_inside_opt.argtypes = [vp, vp, P(C.c_uint8), C.c_int32, vp, C.c_int32,
                                               C.c_float, C.c_int, C.c_int, vp, C.c_int32,
                                               P(C.c_int32)]
    for name in ("cmgpu_scan_batch", "cmgpu_scan_plain"):
        getattr(L, name).argtypes = [vp, vp, C.c_int, C.c_int, P(C.c_uint8), C.c_int64, vp,
                                     C.c_int32, C.c_float, C.c_int, vp, C.c_int32, P(C.c_int32)]
    L.cmgpu_scan_batch_device.argtypes = [vp, vp, C.c_int, C.c_int, vp, C.c_int64, vp, C.c_int32,
                                          C.c_float, C.c_int, vp, C.c_int32, P(C.c_int32)]
    L.cmgpu_vit_filter_build.argtypes = [vp, C.c_int, P(vp)]
    L.cmgpu_vit_filter_free.argtypes = [vp]
    L.cmgpu_vit_filter_free.restype = None
    L.cmgpu_vit_filter_tables.argtypes = [vp, vp, C.c_int32, P(C.c_int32), vp]
    L.cmgpu_vit_score_batch.argtypes = [vp, vp, vp, C.c_int64, vp, C.c_int32, vp, vp]
    L.cmgpu_vit_filter_stats.argtypes = [vp, P(C.c_double), P(C.c_int64), P(C.c_int32)]
    L.cmgpu_msv_filter_build.argtypes = [vp, C.c_int32, C.c_double, C.c_double, C.c_int, P(vp)]
    L.cmgpu_msv_filter_free.argtypes = [vp]
    L.cmgpu_msv_filter_free.restype = None
    L.cmgpu_msv_filter_tables.argtypes = [vp, vp, C.c_int32, P(C.c_int32), vp, vp, vp, vp]
    L.cmgpu_ssv_threshold.argtypes = [vp, C.c_double, P(C.c_int32)]
    L.cmgpu_msv_score_batch.argtypes = [vp, vp, vp, C.c_int64, vp, C.c_int32, vp, vp, vp]
    L.cmgpu_f1_msv_windows.argtypes = [vp, vp, vp, C.c_int64, vp, C.c_int32, C.c_double, C.c_int64, vp,
                                       C.c_int32, P(C.c_int32)]
    L.cmgpu_ssv_diagonals.argtypes = [vp, vp, vp, C.c_int64, vp, C.c_int32, C.c_double, vp, C.c_int32,
                                      P(C.c_int32)]
    L.cmgpu_msv_filter_stats.argtypes = [vp, P(C.c_double), P(C.c_int64), P(C.c_int32)]
    L.cmgpu_prep_cp9.argtypes = [P(CmParams), P(Cp9)]
    L.cmgpu_fwd_filter_build.argtypes = [vp, vp, C.c_double, C.c_double, C.c_int, P(vp)]
    L.cmgpu_fwd_filter_free.argtypes = [vp]
    L.cmgpu_fwd_filter_free.restype = None
    L.cmgpu_fwd_filter_tables.argtypes = [vp, vp, vp, C.c_int32, P(C.c_int32), vp, vp]
    L.cmgpu_fwd_score_batch.argtypes = [vp, vp, vp, C.c_int64, vp, C.c_int32, vp, vp]
    L.cmgpu_f3_filter.argtypes = [vp, vp, vp, vp, vp, C.c_int64, vp, C.c_int32, P(F3Config), vp, C.c_int32,
                                  P(C.c_int32), P(F3Acct)]
    L.cmgpu_fwd_filter_stats.argtypes = [vp, P(C.c_double), P(C.c_int64), P(C.c_int32)]
    L.cmgpu_fwd_filter_set_kernel.argtypes = [vp, C.c_int]
    L.cmgpu_fast_cyk_scan_hb.argtypes = [vp, P(HbBands), vp, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                         P(C.c_float), P(C.c_int64), P(C.c_int64)]
    L.cmgpu_hb_scan_hits.argtypes = [vp, C.c_int, P(HbBands), vp, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                     C.c_float, C.c_int, P(C.c_float), P(C.c_int64), P(C.c_int64), vp, C.c_int32,
                                     P(C.c_int32)]
    L.cmgpu_hb_scan_batch.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, vp, C.c_int64, vp, C.c_int32, vp, vp,
                                      C.c_int64, P(C.c_int64)]
    L.cmgpu_tr_scan_hb.argtypes = [vp, C.c_int, P(TrTables), P(HbBands), vp, vp, vp, vp, vp, C.c_int32, C.c_int32,
                                   C.c_int32, C.c_float, C.c_int, C.c_int, C.c_float, P(C.c_float), P(C.c_int32),
                                   P(C.c_int64), P(C.c_int64), vp, C.c_int32, P(C.c_int32)]
    L.cmgpu_tr_scan_hb_batch.argtypes = [vp, vp, C.c_int, P(TrTables), C.c_int, C.c_int, vp, C.c_int64, vp,
                                         C.c_int32, vp, vp, C.c_int64, P(C.c_int64)]
    L.cmgpu_hb_stats.argtypes = [vp, P(C.c_double), P(C.c_int64), P(C.c_int32)]
    L.cmgpu_tr_qdb_scan.argtypes = [vp, C.c_int, C.c_int, P(TrTables), vp, C.c_int32, C.c_int32, C.c_int32,
                                    C.c_float, C.c_int, C.c_int, P(C.c_float), P(C.c_int32), P(C.c_float), vp,
                                    C.c_int32, P(C.c_int32)]
    L.cmgpu_tr_qdb_scan_batch.argtypes = [vp, vp, C.c_int, C.c_int, P(TrTables), C.c_int, C.c_int, vp, C.c_int64,
                                          vp, C.c_int32, C.c_float, vp, vp, C.c_int64, P(C.c_int64)]
    L.cmgpu_tr_qdb_stats.argtypes = [vp, P(C.c_double), P(C.c_int64), P(C.c_int32)]
    L.cmgpu_tr_qdb_inject_stall.argtypes = [vp, C.c_int32]
    L.cmgpu_tr_qdb_set_deck_budget.argtypes = [vp, C.c_int64]
    L.cmgpu_count_work.argtypes = [P(Cm), C.c_int, C.c_int, C.c_int32, P(C.c_double),
                                   P(C.c_double)]
    L.cmgpu_genomic_sample.argtypes = [C.c_uint32, C.c_int32, C.c_int32, vp]
    L.cmgpu_exp_fit.argtypes = [vp, C.c_int64, C.c_int, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                C.c_double, P(ExpParams)]
    L.cmgpu_calibrate_scan_batch.argtypes = [vp, vp, C.c_int, C.c_int, vp, C.c_int64, vp, C.c_int32, C.c_int, vp,
                                             C.c_int32, P(C.c_int32)]
    L.cmgpu_calibrate.argtypes = [P(CmParams), C.c_int32, C.c_int, P(CalibrateConfig), P(CalibrateResult)]
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != CMGPU_OK:
        raise CmgpuError(rc, lib().cmgpu_last_error().decode(errors="replace"))


# symbols declared in include/cmscan_gpu.h (checked by the CPU test suite)
EXPORTED = [
    "cmgpu_last_error", "cmgpu_version", "cmgpu_prep_configure", "cmgpu_prep_truncated", "cmgpu_ilogsum_table",
    "cmgpu_flogsum_table", "cmgpu_model_upload", "cmgpu_model_free", "cmgpu_workspace_create",
    "cmgpu_workspace_free", "cmgpu_workspace_stats", "cmgpu_workspace_set_shape", "cmgpu_workspace_set_kernel",
    "cmgpu_qdb_scan", "cmgpu_qdb_scan_noalloc", "cmgpu_qdb_scan_cells", "cmgpu_cyk_seq_filter", "cmgpu_final_stage_inside_opt",
    "cmgpu_scan_batch", "cmgpu_scan_batch_device", "cmgpu_scan_plain", "cmgpu_count_work",
    "cmgpu_vit_filter_build", "cmgpu_vit_filter_free", "cmgpu_vit_filter_tables", "cmgpu_vit_score_batch",
    "cmgpu_vit_filter_stats", "cmgpu_msv_filter_build", "cmgpu_msv_filter_free", "cmgpu_msv_filter_tables", "cmgpu_ssv_threshold",
    "cmgpu_msv_score_batch", "cmgpu_f1_msv_windows", "cmgpu_ssv_diagonals", "cmgpu_msv_filter_stats",
    "cmgpu_fast_cyk_scan_hb", "cmgpu_hb_scan_hits", "cmgpu_hb_scan_batch", "cmgpu_hb_stats",
    "cmgpu_tr_scan_hb", "cmgpu_tr_scan_hb_batch", "cmgpu_tr_qdb_scan", "cmgpu_tr_qdb_scan_batch",
    "cmgpu_tr_qdb_stats", "cmgpu_tr_qdb_inject_stall", "cmgpu_tr_qdb_set_deck_budget", "cmgpu_genomic_sample", "cmgpu_exp_fit",
    "cmgpu_calibrate_scan_batch", "cmgpu_calibrate", "cmgpu_fwd_filter_build", "cmgpu_fwd_filter_free",
    "cmgpu_prep_cp9", "cmgpu_fwd_filter_tables", "cmgpu_fwd_score_batch", "cmgpu_f3_filter", "cmgpu_fwd_filter_stats", "cmgpu_fwd_filter_set_kernel",
]
