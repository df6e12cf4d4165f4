"""Regenerates the fixtures in tests/golden/.

* ilogsum_kat.json, state_delta_kat.json: the known answers of the
  reference's own unit tests, parsed from its sources (src/cp9.rs tests
  `ilogsum_sentinel_and_bounds`, `ilogsum_table_matches_c_dump`,
  `ilogsum_table_endpoints_match_c_formula`; src/cm_qdband.rs
  `test_state_delta`).  Needs the reference checkout: set REFERENCE_ROOT to
  its path; run it only where that exists.
* genomic_kat.json: the random genomic sequences of cmcalibrate's generator
  for seed 181 that the reference's test `rng_sample_matches_c` pins against
  C Infernal (src/cm_calibrate.rs:1253-1268).
* cm_file_kat.json: the two model texts of the reference's CM reader tests
  (`test_minimal_cm_parse`, `test_v1_1_cm_parse`, src/cm_file.rs:2155-2212)
  with the name / states / nodes / clen those tests assert.
* pipeline_kat.json: the filter thresholds per database size that the
  reference's `thresholds_match_c_table` test asserts
  (src/cm_pipeline.rs:2170-2187).
* histogram_kat.json: the exponential tail fit of the reference's
  `test_cmcalibrate_sequence` (src/easel/histogram.rs:543-586), whose mu and
  lambda the reference pins to a probe of C libeasel.
* tmap_kat.json: the CM transition map (cm_create_transition_map,
  src/cp9.rs:480-740), which state occupancy and the CP9 subpath sums index.
* scan_small.json: the oracle's hits on one fixed seeded model and sequence,
  a regression lock for the oracle itself.

Usage: REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden.py
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("REFERENCE_ROOT")


def ilogsum_kats():
    src = open(os.path.join(REF, "src", "cp9.rs")).read()
    body = src[src.index("fn ilogsum_table_matches_c_dump"):]
    body = body[: body.index("}\n\n")]
    table = [[int(a), int(b)] for a, b in re.findall(r"\((\d+),\s*(\d+)\)", body)]
    calls = []
    sent = src[src.index("fn ilogsum_sentinel_and_bounds"):]
    sent = sent[: sent.index("}\n\n")]
    end = src[src.index("fn ilogsum_table_endpoints_match_c_formula"):]
    end = end[: end.index("}\n}")]
    for blk in (sent, end):
        for a, b, w in re.findall(r"assert_eq!\(ilogsum\(([^,]+),\s*([^)]+)\),\s*([^)]+)\)", blk):
            def val(x):
                x = x.strip()
                return -987654321 if x == "-INFTY" else int(x)
            calls.append([val(a), val(b), val(w)])
    return {"source": "src/cp9.rs:81-117", "table": table, "calls": calls}


def state_delta_kats():
    src = open(os.path.join(REF, "src", "cm_qdband.rs")).read()
    body = src[src.index("fn test_state_delta()"):]
    body = body[: body.index("}\n")]
    codes = {"D_ST": 0, "MP_ST": 1, "ML_ST": 2, "MR_ST": 3, "IL_ST": 4, "IR_ST": 5, "S_ST": 6,
             "E_ST": 7, "B_ST": 8, "EL_ST": 9}
    pairs = [[codes[s], int(d)] for s, d in re.findall(r"state_delta\((\w+)\),\s*(\d+)", body)]
    return {"source": "src/cm_qdband.rs:639-652", "state_delta": pairs}


def genomic_kats():
    src = open(os.path.join(REF, "src", "cm_calibrate.rs")).read()
    body = src[src.index("fn rng_sample_matches_c"):]
    body = body[: body.index("}\n")]
    seed = int(re.search(r"EslRandom::new\((\d+)\)", body).group(1))
    length = int(re.search(r"sample_genomic_sequence_from_hmm\(&mut r, &ghmm, (\d+)\)", body).group(1))
    seqs = re.findall(r'assert_eq!\(d\d, "([0-3]+)"\)', body)
    return {"source": "src/cm_calibrate.rs:1253-1268", "seed": seed, "L": length, "sequences": seqs}


def cm_file_kats():
    src = open(os.path.join(REF, "src", "cm_file.rs")).read()
    out = []
    for test in ("fn test_minimal_cm_parse", "fn test_v1_1_cm_parse"):
        body = src[src.index(test):]
        body = body[: body.index("\n    }\n")]
        text = re.search(r'let cm_text = r#"(.*?)"#;', body, re.S).group(1)
        want = dict(re.findall(r"assert_eq!\(cm\.(\w+), ([^)]+)\);", body))
        out.append({"test": test[3:], "text": text, "name": want["name"].strip('"'), "M": int(want["m"]),
                    "nodes": int(want["nodes"]), "clen": int(want["clen"])})
    return {"source": "src/cm_file.rs:2155-2212", "models": out}


def pipeline_kats():
    src = open(os.path.join(REF, "src", "cm_pipeline.rs")).read()
    body = src[src.index("fn thresholds_match_c_table"):]
    body = body[: body.index("\n    }\n")]
    cases = []
    for blk in body.split("let p = CmPipeline::new_default(")[1:]:
        z = float(blk[: blk.index(")")])
        want = {}
        for k, v in re.findall(r"assert_eq!\(p\.(\w+), ([0-9.e-]+)\);", blk):
            want[k] = float(v)
        for neg, k in re.findall(r"assert!\((!?)p\.(\w+)\);", blk):
            want[k] = not neg
        cases.append({"z": z, "want": want})
    return {"source": "src/cm_pipeline.rs:2170-2187", "cases": cases}


def histogram_kats():
    src = open(os.path.join(REF, "src", "easel", "histogram.rs")).read()
    body = src[src.index("fn test_cmcalibrate_sequence"):]
    body = body[: body.index("\n    }\n")]
    scores = [float(x) for x in re.search(r"let scores = \[(.*?)\];", body, re.S).group(1).replace("\n", " ").split(",")
              if x.strip()]
    mass = float(re.search(r"get_tail_by_mass\(([0-9.]+)\)", body).group(1))
    mu = re.search(r"assert_eq!\(mu, ([0-9.e-]+)\);", body).group(1)
    lam = re.search(r"assert_eq!\(lambda, ([0-9.e-]+)\);", body).group(1)
    return {"source": "src/easel/histogram.rs:543-586", "scores": scores, "tail_mass": mass, "mu": mu,
            "lambda": lam}


def tmap_kats():
    """cm_create_transition_map's table (src/cp9.rs:480-740) as
    [parent unique state, node type, child unique state, transition]."""
    src = open(os.path.join(REF, "src", "cp9.rs")).read()
    body = src[src.index("pub fn cm_create_transition_map"):]
    body = body[: body.index("\n}\n")]
    ids = {"ROOT_S": 0, "ROOT_IL": 1, "ROOT_IR": 2, "BEGL_S": 3, "BEGR_S": 4, "BEGR_IL": 5, "MATP_MP": 6,
           "MATP_ML": 7, "MATP_MR": 8, "MATP_D": 9, "MATP_IL": 10, "MATP_IR": 11, "MATL_ML": 12, "MATL_D": 13,
           "MATL_IL": 14, "MATR_MR": 15, "MATR_D": 16, "MATR_IR": 17, "BIF_B": 18, "END_E": 19}
    nds = {"BIF_ND": 0, "MATP_ND": 1, "MATL_ND": 2, "MATR_ND": 3, "BEGL_ND": 4, "BEGR_ND": 5, "ROOT_ND": 6,
           "END_ND": 7}
    rows = [[ids[a], nds[b], ids[c], int(n)] for a, b, c, n in
            re.findall(r"tmap\[(\w+) as usize\]\[(\w+) as usize\]\[(\w+) as usize\] = (\d+);", body)]
    return {"source": "src/cp9.rs:480-740", "entries": rows}


def scan_small():
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    from helpers import frame, models, planted_seq
    name, n, nplant, seed = "small2", 1500, 2, 77
    cm, g, l = models(name)
    dsq = frame(planted_seq(cm, n, 0.5, nplant, seed=seed))
    cases = []
    for sr, band, cutoff in ((0, 1, 0.0), (1, 2, 0.0), (1, 0, 2.0)):
        hits, _, _, _ = oracle.qdb_scan(l, sr, band, dsq, 1, n, cutoff, True)
        cases.append({"semiring": sr, "band": band, "cutoff": cutoff,
                      "hits": [[h[0], h[1], round(h[2], 4), round(h[3], 6)] for h in hits]})
    return {"model": name, "local": True, "n": n, "nplant": nplant, "seed": seed, "cases": cases}


def main():
    if not REF or not os.path.isdir(REF):
        print("REFERENCE_ROOT is not set to a reference checkout: only scan_small.json is regenerated")
    else:
        with open(os.path.join(HERE, "ilogsum_kat.json"), "w") as f:
            json.dump(ilogsum_kats(), f, indent=1)
        with open(os.path.join(HERE, "state_delta_kat.json"), "w") as f:
            json.dump(state_delta_kats(), f, indent=1)
        with open(os.path.join(HERE, "genomic_kat.json"), "w") as f:
            json.dump(genomic_kats(), f, indent=1)
        with open(os.path.join(HERE, "cm_file_kat.json"), "w") as f:
            json.dump(cm_file_kats(), f, indent=1)
        with open(os.path.join(HERE, "pipeline_kat.json"), "w") as f:
            json.dump(pipeline_kats(), f, indent=1)
        with open(os.path.join(HERE, "histogram_kat.json"), "w") as f:
            json.dump(histogram_kats(), f, indent=1)
        with open(os.path.join(HERE, "tmap_kat.json"), "w") as f:
            json.dump(tmap_kats(), f)
    with open(os.path.join(HERE, "scan_small.json"), "w") as f:
        json.dump(scan_small(), f, indent=1)


if __name__ == "__main__":
    main()
