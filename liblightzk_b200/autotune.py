"""Measured autotuner for the library's tuning table (lzk_tune_set).

Per size class 2^log_n it times candidates on the device (CUDA events,
seeded random inputs, median of a few runs) and installs the fastest:

  window  Pippenger window width of plain-base MSMs (the cost model's
          width and its neighbours)
  chunk   sorted bucket entries one accumulation thread adds (32, 64, 128)
  run     buckets per lane run in the bucket-reduction tiles (4, 8, 16)
  ntt     elements per block of an NTT pass, i.e. how a transform's stages
          split into passes (1024, 2048, 4096)
  table_*  window width, chunk and run of MSMs over shifted-copy tables
          (provers, batch plans with fixed bases)

Every autotuned MSM, batch plan and prover made afterwards uses the table
(a prover or plan reads it when it is created).  `save` / `load` keep a
table as JSON, so a tuned table can be reused without re-timing.
"""
import json
import os

import numpy as np
import torch

from . import _capi, msm, ntt, synth

# measured tables shipped with the package, by GPU name
DEFAULT_TABLES = {"B200": os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning", "b200.json")}

WINDOW, CHUNK, RUN, NTT_BLOCK, TABLE_WINDOW, TABLE_CHUNK, TABLE_RUN = range(7)
KNOBS = {"window": WINDOW, "chunk": CHUNK, "run": RUN, "ntt": NTT_BLOCK, "table_window": TABLE_WINDOW,
         "table_chunk": TABLE_CHUNK, "table_run": TABLE_RUN}


def _time(fn, reps):
    ts = []
    for _ in range(reps + 1):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts[1:]))


def set_value(knob, group, log_n, value):
    _capi.call("lzk_tune_set", KNOBS[knob], group, log_n, value)


def get_value(knob, group, log_n):
    return int(_capi.lib().lzk_tune_get(KNOBS[knob], group, log_n))


def tune(group=1, log_ns=range(10, 21), spread=2, reps=3, seed=11, install=True):
    """window widths only: {log_n: (best_c, {c: ms})}"""
    table = {}
    top = max(log_ns)
    sc_all = synth.random_fr(1 << top, seed, 90)
    bases_all = synth.fixed_base(group, synth.random_fr(1 << top, seed, 91))
    for lg in log_ns:
        n = 1 << lg
        set_value("window", group, lg, 0)      # model value as the centre
        c0 = msm.autotune_window(group, n)
        res = {}
        for c in range(max(2, c0 - spread), min(22, c0 + spread) + 1):
            res[c] = _time(lambda c=c: msm.msm(group, sc_all[:n], bases_all[:n], window_bits=c), reps)
        best = min(res, key=res.get)
        table[lg] = (best, res)
        if install:
            set_value("window", group, lg, best)
    return table


def tune_msm(group=1, log_ns=range(10, 21), spread=2, reps=3, seed=11, chunks=(32, 64, 128), runs=(4, 8, 16)):
    """per size class: window width and reduction run together (the run
    sets how much each bucket costs, which moves the best width), then the
    accumulation chunk at that pair; installs them and returns
    {log_n: {"window": best_c, "run": best_run, "chunk": best_chunk,
             "ms": {"c,run": ms}, "chunk_ms": {chunk: ms}}}"""
    out = {}
    top = max(log_ns)
    sc_all = synth.random_fr(1 << top, seed, 90)
    bases_all = synth.fixed_base(group, synth.random_fr(1 << top, seed, 91))
    for lg in log_ns:
        n = 1 << lg
        s, b = sc_all[:n], bases_all[:n]
        for k in ("window", "chunk", "run"):
            set_value(k, group, lg, 0)
        c0 = msm.autotune_window(group, n)
        res = {}
        for c in range(max(2, c0 - spread), min(22, c0 + spread) + 1):
            for r in runs:
                set_value("run", group, lg, r)
                res[(c, r)] = _time(lambda c=c: msm.msm(group, s, b, window_bits=c), reps)
        c_best, r_best = min(res, key=res.get)
        set_value("window", group, lg, c_best)
        set_value("run", group, lg, r_best)
        cres = {}
        for v in chunks:
            set_value("chunk", group, lg, v)
            cres[v] = _time(lambda: msm.msm(group, s, b), reps)
        ch_best = min(cres, key=cres.get)
        set_value("chunk", group, lg, ch_best)
        out[lg] = {"window": c_best, "run": r_best, "chunk": ch_best,
                   "ms": {f"{c},{r}": v for (c, r), v in res.items()}, "chunk_ms": cres}
    return out


def tune_msm_table(group=1, log_ns=range(10, 21), spread=(4, 2), reps=3, seed=11, runs=(4, 8, 16), chunks=(32, 64, 128)):
    """window width and reduction run (together), then chunk, of an MSM over
    a shifted-copy table, per size class, timing one MSM of 2^log_n points
    (the table of each width built outside the timing; widths from
    spread[0] below the cost model's to spread[1] above); installs the best
    and returns {log_n: {"window", "run", "chunk", "ms": {"c,run": ms},
    "chunk_ms": {chunk: ms}}}"""
    out = {}
    top = max(log_ns)
    sc_all = synth.random_fr(1 << top, seed, 94)
    bases_all = synth.fixed_base(group, synth.random_fr(1 << top, seed, 95))
    for lg in log_ns:
        n = 1 << lg
        s, b = sc_all[:n], bases_all[:n]
        for knob in ("table_window", "table_run", "table_chunk"):
            set_value(knob, group, lg, 0)
        c0 = msm.autotune_window(group, n, precomputed=True)
        res, tabs = {}, {}
        # the model leans to wide windows (it undercounts the bucket
        # reduction), so the candidates reach further below it than above
        for c in range(max(4, c0 - spread[0]), min(20, c0 + spread[1]) + 1):
            w = msm.windows_for(c)
            tabs[c] = msm.precompute(group, b, c, w, n)
            for r in runs:
                set_value("table_run", group, lg, r)
                res[(c, r)] = _time(lambda c=c, w=w: msm.msm_precomputed(group, s, tabs[c], c, w, n), reps)
        c_best, r_best = min(res, key=res.get)
        set_value("table_window", group, lg, c_best)
        set_value("table_run", group, lg, r_best)
        w = msm.windows_for(c_best)
        cres = {}
        for v in chunks:
            set_value("table_chunk", group, lg, v)
            cres[v] = _time(lambda: msm.msm_precomputed(group, s, tabs[c_best], c_best, w, n), reps)
        ch_best = min(cres, key=cres.get)
        set_value("table_chunk", group, lg, ch_best)
        del tabs
        out[lg] = {"window": c_best, "run": r_best, "chunk": ch_best,
                   "ms": {f"{c},{r}": v for (c, r), v in res.items()}, "chunk_ms": cres}
    return out


def tune_ntt(log_ns=range(12, 23), reps=3, seed=12, blocks=(1024, 2048, 4096), direction=ntt.COSET_FORWARD):
    """NTT block size per transform size; installs the fastest and returns
    {log_n: (best, {block: ms})}"""
    out = {}
    for lg in log_ns:
        x = synth.random_fr(1 << lg, seed, 92)
        ntt.prepare(lg)
        res = {}
        for v in blocks:
            set_value("ntt", 0, lg, v)
            res[v] = _time(lambda: ntt.ntt(x, lg, direction), reps)
        best = min(res, key=res.get)
        set_value("ntt", 0, lg, best)
        out[lg] = (best, res)
    return out


def tune_prover(circuit, pk, mode=0, window_bits=17, chunks=(32, 64), runs=(4, 8, 16), proofs=8, seed=13):
    """accumulation chunk and reduction run of a Groth16 prover's own MSMs
    (shifted-table MSMs over the circuit's variables, the L + H concatenation
    and the G2 query), chosen by timing whole proofs; installs the best
    pair for those size classes and returns {(chunk, run): ms per proof}"""
    from . import device, groth16
    z = circuit.witness(seed)
    rs = device.to_host(synth.random_fr(2, seed, 93))
    nl = circuit.n_vars - circuit.n_public - 1
    classes = {1: {int(np.ceil(np.log2(circuit.n_vars))), int(np.ceil(np.log2(nl + circuit.M - 1)))},
               2: {int(np.ceil(np.log2(circuit.n_vars)))}}

    def install(chunk, run):
        for g, lgs in classes.items():
            for lg in lgs:
                set_value("table_chunk", g, lg, chunk)
                set_value("table_run", g, lg, run)

    res = {}
    for chunk in chunks:
        for run in runs:
            install(chunk, run)
            p = groth16.Prover(circuit, pk, mode=mode, window_bits=window_bits)
            res[(chunk, run)] = _time(lambda: [p.prove(z, rs[0], rs[1]) for _ in range(proofs)], 2) / proofs
            p.close()
    best = min(res, key=res.get)
    install(*best)
    return res


def load_default():
    """install the packaged table measured on this GPU model, if there is
    one; returns its path or None"""
    name = torch.cuda.get_device_name()
    for key, path in DEFAULT_TABLES.items():
        if key in name and os.path.exists(path):
            load(path)
            return path
    return None


def current(groups=(1, 2), log_ns=range(0, 33)):
    """the installed table as a JSON-able dict of non-default entries"""
    t = {"msm": {}, "ntt": {}}
    for g in groups:
        t["msm"][str(g)] = {k: {str(lg): get_value(k, g, lg) for lg in log_ns}
                            for k in ("window", "chunk", "run", "table_window", "table_chunk", "table_run")}
    t["ntt"] = {str(lg): get_value("ntt", 0, lg) for lg in log_ns}
    return t


def save(path, table=None):
    with open(path, "w") as f:
        json.dump(table or current(), f, indent=1, sort_keys=True)


def load(path):
    """install a table written by save()"""
    t = json.load(open(path))
    for g, knobs in t.get("msm", {}).items():
        for k, vals in knobs.items():
            for lg, v in vals.items():
                set_value(k, int(g), int(lg), int(v))
    for lg, v in t.get("ntt", {}).items():
        set_value("ntt", 0, int(lg), int(v))
