"""cmcalibrate on the GPU (src/cm_calibrate.rs), mirroring the reference's
functions by name.

calibrate_cm(cm, cfg) runs the whole calibration in the library
(cmgpu_calibrate): N = round(L_Mb * 1e6 / 10 kb) random genomic sequences
from the reference's generator, the glocal and local configurations with
both QDB band sets at cfg.beta, ONE batched GPU scan per exp mode (glocal /
local x CYK / Inside) with cutoff -inf, and the exponential tail fit of each
mode.  The pieces are exposed for tests and callers that bring their own
sequences: sample_genomic_sequences, collect_scores, fit_histogram.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _native as N
from . import model as Mdl
from .scan import CYK_F32, INSIDE_I32, QDB2, Scanner

EXP_CM_GC, EXP_CM_GI, EXP_CM_LC, EXP_CM_LI = 0, 1, 2, 3
EXP_NMODES = 4
EXPTAIL_CHUNKLEN = 10000
MODE_NAMES = ("GC", "GI", "LC", "LI")


def exp_mode_is_local(m: int) -> bool:
    return m in (EXP_CM_LC, EXP_CM_LI)


def exp_mode_is_inside(m: int) -> bool:
    return m in (EXP_CM_GI, EXP_CM_LI)


@dataclass
class CalibrateConfig:
    """CalibrateConfig (src/cm_calibrate.rs:1048-1075) with its defaults."""
    seed: int = 181
    l_mb: float = 1.6
    beta: float = 1e-15
    nonbanded: bool = False
    gtailn: int = 250
    ltailn: int = 750
    tailp: Optional[float] = None
    do_null3: bool = True

    def as_struct(self) -> N.CalibrateConfig:
        return N.CalibrateConfig(self.seed, self.l_mb, self.beta, int(self.nonbanded), self.gtailn, self.ltailn,
                                 float(self.tailp) if self.tailp else 0.0, int(self.do_null3))


def n_sequences(cfg: CalibrateConfig) -> int:
    """N = round(L_Mb * 1e6 / chunk) (src/cm_calibrate.rs:1105-1109)."""
    return int(((cfg.l_mb * 1_000_000.0) / float(np.float32(EXPTAIL_CHUNKLEN))) + 0.5)


def _exp_dict(e: N.ExpParams) -> dict:
    return dict(lambda_=e.lambda_, mu=e.mu, dbsize=e.dbsize, nrandhits=e.nrandhits, mu_orig=e.mu_orig,
                tailp=e.tailp)


def sample_genomic_sequences(seed: int, L: int, nseq: int) -> np.ndarray:
    """generate_sequences: nseq frames [255, L residues, 255] back to back."""
    out = np.zeros(nseq * (L + 2), np.uint8)
    N.check(N.lib().cmgpu_genomic_sample(int(seed), int(L), int(nseq), out.ctypes.data))
    return out


def calibration_configs(cm: Mdl.SynthCM, W: int, cfg: CalibrateConfig):
    """The glocal and local CMs calibrate_cm scans (src/cm_calibrate.rs:
    1128-1148): both band sets at cfg.beta on the global transitions, the
    model's W kept; full bands with cfg.nonbanded."""
    out = []
    for local in (False, True):
        c = Mdl.configure(cm, local=local, W=W, beta1=cfg.beta, beta2=cfg.beta)
        if cfg.nonbanded:
            for k in ("dmin1", "dmin2"):
                getattr(c, k)[:] = 0
            for k in ("dmax1", "dmax2"):
                getattr(c, k)[:] = c.W
        out.append(c)
    return tuple(out)


def collect_scores(sc: Scanner, inside: bool, frames: np.ndarray, windows: np.ndarray, do_null3: bool) -> np.ndarray:
    """collect_scores (src/cm_calibrate.rs:953-989): the kept hits of every
    window (BATCH_HIT_DTYPE, window order) of one mode's batched scan."""
    return sc.calibrate_scan_batch(INSIDE_I32 if inside else CYK_F32, QDB2, frames, windows, do_null3)


def fit_histogram(scores, exp_mode: int, n_seqs: int, L: int, gtailn: int = 250, ltailn: int = 750,
                  tailp: Optional[float] = None, dbsize: float = 0.0) -> dict:
    """fit_histogram + set_exp_info (src/cm_calibrate.rs:1000-1099)."""
    s = np.ascontiguousarray(scores, np.float32)
    e = N.ExpParams()
    N.check(N.lib().cmgpu_exp_fit(s.ctypes.data, len(s), exp_mode, n_seqs, L, gtailn, ltailn,
                                  float(tailp) if tailp else 0.0, float(dbsize), C.byref(e)))
    return _exp_dict(e)


def calibrate_cm(cm: Mdl.SynthCM, cfg: Optional[CalibrateConfig] = None, W: Optional[int] = None,
                 device: int = 0) -> dict:
    """calibrate_cm (src/cm_calibrate.rs:1102-1182) on the GPU.  W defaults
    to the model's W at beta_W = 1e-7.  Returns exp[mode] (lambda_, mu =
    extrapolated, mu_orig, tailp, nrandhits, dbsize), nhits, dbsize, and the
    scans' cells and device time."""
    cfg = cfg or CalibrateConfig()
    if W is None:
        W = Mdl.configure(cm, local=False).W
    p, keep = Mdl.params_struct(cm)
    r = N.CalibrateResult()
    cs = cfg.as_struct()
    N.check(N.lib().cmgpu_calibrate(C.byref(p), int(W), int(device), C.byref(cs), C.byref(r)))
    del keep
    return dict(exp=[_exp_dict(r.exp[m]) for m in range(EXP_NMODES)], nhits=list(r.nhits), dbsize=r.dbsize,
                cells=r.cells, terms=r.terms, kernel_ms=r.kernel_ms, launches=r.launches)
