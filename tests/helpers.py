"""Shared seeded inputs for the parity tests."""
import numpy as np

from infernox_b200 import model, synth


def frame(seq: np.ndarray) -> np.ndarray:
    return np.concatenate([[255], np.asarray(seq, np.uint8), [255]]).astype(np.uint8)


def planted_seq(cm, n: int, gc: float, nplant: int, seed: int, degenerate: float = 0.0):
    """i.i.d. background with `nplant` sampled homologs at seeded positions;
    a fraction of residues may be replaced by IUPAC codes 5..15."""
    rng = np.random.default_rng(seed)
    seq = synth.random_dsq(n, gc, rng)
    for _ in range(nplant):
        h = synth.emit(cm, rng)
        if len(h) == 0 or len(h) >= n:
            continue
        pos = int(rng.integers(0, n - len(h)))
        seq[pos:pos + len(h)] = h
    if degenerate > 0:
        m = rng.random(n) < degenerate
        seq[m] = rng.integers(5, 16, m.sum()).astype(np.uint8)
    return seq


_cache = {}


def models(name: str):
    """(synthetic cm, global configured, local configured) by name, cached."""
    if name in _cache:
        return _cache[name]
    if name == "trna":
        cm = synth.synth_cm(synth.trna_like(), 11, name=name)
    elif name == "small0":
        cm = synth.synth_cm(synth.structure(30, 0.4, 0, 3), 21, name=name)
    elif name == "small2":
        cm = synth.synth_cm(synth.structure(48, 0.45, 2, 4), 22, name=name)
    elif name == "cfg2":
        cm = synth.synth_cm(synth.structure(120, 0.5, 3, 5), 23, name=name)
    elif name == "mb3":
        cm = synth.synth_cm(synth.structure(90, 0.4, 3, 6, layout="multibranch"), 24, name=name)
    elif name == "cfg0":
        # the --nohmm CYK workload's model shape: 72 columns, a 7 bp closing
        # stem around three 5 bp hairpins (a 4-stem multibranch)
        cm = synth.synth_cm(synth.trna_like(), 11, name=name)
    elif name == "cfg3":
        # the bifurcation-heavy truncated workload's model shape: 1500
        # columns, 60% paired, 25 bifurcations
        cm = synth.synth_cm(synth.structure(1500, 0.6, 25, 31), 33, name=name)
    else:
        raise KeyError(name)
    r = (cm, model.configure(cm, local=False), model.configure(cm, local=True))
    _cache[name] = r
    return r


_ocache = {}


def oracle_cfg(name: str, local: bool):
    """The model configured from the oracle's own table builders
    (oracle/prep_oracle.c) instead of the library's: the oracle side of a
    parity test then shares no table with the GPU side."""
    key = (name, local)
    if key in _ocache:
        return _ocache[key]
    import oracle
    from infernox_b200.model import ConfiguredCM
    cm, g, l = models(name)
    t = oracle.prep_configure(cm, local)
    c = ConfiguredCM(
        name=cm.name, M=cm.M, W=t["W"], flags=t["flags"], clen=cm.clen,
        sttype=np.ascontiguousarray(cm.st.sttype, np.int8), stid=np.ascontiguousarray(cm.st.stid, np.int8),
        cfirst=np.ascontiguousarray(cm.st.cfirst, np.int32), cnum=np.ascontiguousarray(cm.st.cnum, np.int32),
        el_selfsc=t["el_selfsc"], iel_selfsc=t["iel_selfsc"], null=np.asarray(cm.null, np.float32),
        n3_omega=float(np.float32(cm.n3_omega)),
        **{k: t[k] for k in ("tsc", "oesc", "endsc", "beginsc", "itsc", "ioesc", "iendsc", "ibeginsc",
                             "dmin1", "dmax1", "dmin2", "dmax2", "t_local")})
    _ocache[key] = c
    return c
