"""The whole-solve graph's Picard-loop decisions (CPU): the __host__ __device__ functions of
csrc/ssa_state.h, which the graph's control kernels run, compiled here with g++ and driven
through seeded scenarios, against a restatement of the host loop they replace
(picard_manager and linear_solve_mixed in csrc/ssa_capi.cu; SSAFD.cc:962-1119).  Each
scenario draws the linear solves' outcomes, zero-diagonal markers and nu*H norms; both
sides must choose the same KSP tolerances, stop at the same point with the same status,
and count the same iterations, refinement steps and loop passes."""
import json
import math
import os
import shutil
import subprocess

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OK, EKSP, EPICARD, EZERODIAG, ENAN = 0, 4, 5, 6, 7
KSP_OK, KSP_MAXIT, KSP_BREAKDOWN, KSP_NAN, KSP_STALLED, KSP_OUTER_DONE = 0, -3, -5, -7, -11, 1


def _header_codes():
    text = open(os.path.join(REPO, "include", "pism_ssa_gpu.h")).read()
    import re
    return {m.group(1): int(m.group(2)) for m in re.finditer(r"\b(PISM_GPU_SSA_E?\w+)\s*=\s*(\d+)", text)}


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    exe = str(tmp_path_factory.mktemp("pc") / "check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(REPO, "include"), "-I",
                    os.path.join(REPO, "pismv0.7.3_b200", "csrc"),
                    os.path.join(REPO, "tests", "picard_control_check.cc"), "-o", exe], check=True)
    return exe


def test_status_codes_match_the_header():
    codes = _header_codes()
    assert (codes["PISM_GPU_SSA_OK"], codes["PISM_GPU_SSA_EKSP"], codes["PISM_GPU_SSA_EPICARD"],
            codes["PISM_GPU_SSA_EZERODIAG"], codes["PISM_GPU_SSA_ENAN"]) == (OK, EKSP, EPICARD, EZERODIAG, ENAN)


# ---- the host loop, restated ----

def host_mixed(records, max_refine):
    """linear_solve_mixed's refinement loop over inner-solve records (iter, status, r2, b2)."""
    inner, status, steps, final, used = 0, KSP_OK, 0, None, 0
    refine = 0
    while True:
        it, st, r2, b2 = records[used]
        used += 1
        rn, bn = math.sqrt(r2), math.sqrt(b2)
        final = rn / bn if bn > 0 else rn
        if not math.isfinite(rn):
            status = KSP_NAN
            break
        if st == KSP_OUTER_DONE:
            break
        if refine >= max_refine:
            status = KSP_MAXIT
            break
        inner += it
        steps += 1
        if st in (KSP_NAN, KSP_STALLED):
            status = st
            break
        if it == 0:
            status = KSP_BREAKDOWN
            break
        refine += 1
    return inner, status, steps, final, used


def host_picard(c, iters, mixed, max_refine, rebuilds=None):
    """picard_manager: returns status, Picard iterations, KSP total, refinement steps, rtols;
    `rebuilds` (a list) gets, per Picard pass, whether it rebuilds the coarse levels"""
    last, ksp_total, steps, rtols, k_done = 1.0, 0, 0, [], 0
    acc = 0.0
    rebuilds = rebuilds if rebuilds is not None else []
    for k in range(c["max_it"]):
        due = k == 0 or not (c["lag"] > 0.0) or acc >= c["lag"]
        if due:
            acc = 0.0
        rebuilds.append(1 if due else 0)
        rtol = c["ksp_rtol"]
        if c["adaptive"] and last >= 2.0 * c["tol"]:
            rtol = min(c["max"], max(c["ksp_rtol"], c["factor"] * last))
        rtols.append(rtol)
        rec = iters[k]
        if mixed:
            its, status, st_steps, _, used = host_mixed(rec["refine"], max_refine)
            steps += st_steps
            rec["used"] = used
        else:
            its, status = rec["iter"], rec["status"]
        ksp_total += its
        if rec["zd"] >= 0:
            return EZERODIAG, k_done, ksp_total, steps, rtols
        if status != KSP_OK:
            return EKSP, k_done, ksp_total, steps, rtols
        norm, change = rec["norm"], rec["change"]
        if norm > 0 and math.isfinite(norm) and math.isfinite(change):
            acc += change / norm
        k_done = k + 1
        if not (math.isfinite(norm) and math.isfinite(change)):
            return ENAN, k_done, ksp_total, steps, rtols
        if norm == 0 or (change / norm < c["tol"] and rtol <= c["ksp_rtol"]):
            return OK, k_done, ksp_total, steps, rtols
        last = change / norm if norm > 0 else 0.0
    return EPICARD, k_done, ksp_total, steps, rtols


# ---- seeded scenarios ----

def scenario(seed, mixed):
    rng = np.random.default_rng(seed)
    c = {"adaptive": int(rng.random() < 0.7), "ksp_rtol": float(10.0 ** rng.uniform(-10, -5)),
         "max": float(10.0 ** rng.uniform(-3, -1)), "factor": float(rng.choice([0.1, 0.5, 1.0, 2.0])),
         "tol": float(10.0 ** rng.uniform(-6, -3)), "max_it": int(rng.integers(3, 40)),
         "lag": float(rng.choice([0.0, 0.0, 1e-3, 1e-2, 0.1, 0.5]))}
    c["max"] = max(c["max"], c["ksp_rtol"])
    max_refine = int(rng.integers(2, 8))
    clean = seed % 2 == 0   # even seeds: no injected failures, a contracting Picard iteration
    change_rel = 10.0 ** rng.uniform(-1, 0)
    decay = rng.uniform(0.3, 0.7) if clean else rng.uniform(0.3, 0.95)
    iters = []
    for k in range(c["max_it"]):
        rec = {"zd": -1, "norm": float(rng.uniform(1e3, 1e5))}
        rec["change"] = rec["norm"] * change_rel * decay ** k
        u = 1.0 if clean else rng.random()
        if u < 0.02:
            rec["zd"] = int(rng.integers(0, 1000))
        elif u < 0.04:
            rec["norm"] = float("nan")
        elif u < 0.05:
            rec["norm"] = 0.0
        if mixed:
            recs = []
            for _ in range(max_refine + 2):
                v = rng.uniform(0.3, 1.0) if clean else rng.random()
                b2 = float(rng.uniform(1.0, 10.0))
                r2 = b2 * float(10.0 ** rng.uniform(-16, -2))
                if v < 0.25:
                    recs.append((0, KSP_OUTER_DONE, r2, b2))
                elif v < 0.27:
                    recs.append((int(rng.integers(1, 9)), KSP_NAN if v < 0.26 else KSP_STALLED, r2, b2))
                elif v < 0.29:
                    recs.append((0, KSP_OK, r2, b2))
                elif v < 0.30:
                    recs.append((3, KSP_OK, float("nan"), b2))
                else:
                    recs.append((int(rng.integers(1, 12)), KSP_OK, r2, b2))
            if clean:   # the outer test met within the refinement budget
                recs = recs[:int(rng.integers(0, max_refine))]
            recs.append((0, KSP_OUTER_DONE, 1e-30, 1.0))
            rec["refine"] = recs
        else:
            rec["iter"] = int(rng.integers(0, 200))
            rec["status"] = KSP_OK if clean else int(rng.choice([KSP_OK] * 30 + [KSP_MAXIT, KSP_NAN, KSP_BREAKDOWN, KSP_STALLED]))
            rec["r2"], rec["b2"] = float(rng.uniform(0, 1e-12)), float(rng.uniform(1, 10))
        iters.append(rec)
    return c, max_refine, iters


def run_device(driver, c, iters, mixed, max_refine):
    """The graph's sequence of control steps, fed the records the host loop consumed."""
    lines = ["const %d %r %r %r %r %d %r" % (c["adaptive"], c["ksp_rtol"], c["max"], c["factor"], c["tol"],
                                              c["max_it"], c["lag"]),
             "start"]
    marks = []   # what each print checks
    for k, rec in enumerate(iters):
        lines += ["begin", "print"]
        marks.append(("begin", k))
        if mixed:
            for q in range(rec.get("used", 0)):
                it, st, r2, b2 = rec["refine"][q]
                lines += ["refine_end %d %d %r %r %d" % (it, st, r2, b2, max_refine), "print"]
                marks.append(("refine", k, q, rec["used"]))
        else:
            lines += ["ksp_end %d %d %r %r 4" % (rec["iter"], rec["status"], rec["r2"], rec["b2"]), "print"]
            marks.append(("ksp", k))
        lines += ["after %d" % rec["zd"], "print"]
        marks.append(("after", k))
        lines += ["test %r %r" % (rec["norm"], rec["change"]), "print"]
        marks.append(("test", k))
    out = subprocess.run([driver], input="\n".join(lines) + "\n", capture_output=True, text=True, check=True)
    return [json.loads(l) for l in out.stdout.splitlines()], marks


@pytest.mark.parametrize("mixed", [False, True])
@pytest.mark.parametrize("seed", range(40))
def test_device_decisions_equal_the_host_loop(driver, seed, mixed):
    c, max_refine, iters = scenario(seed, mixed)
    rebuilds = []
    status, k_done, ksp_total, steps, rtols = host_picard(c, iters, mixed, max_refine, rebuilds)
    n_iters = len(rtols)
    states, marks = run_device(driver, c, iters[:n_iters], mixed, max_refine)
    # the graph stops where the host loop stops: not done before the last Picard pass
    last = None
    for st, mark in zip(states, marks):
        kind, k = mark[0], mark[1]
        if kind == "begin":
            assert st["rtol"] == rtols[k], (k, st["rtol"], rtols[k])
            assert st["passes"] == k + 1
            assert st["rebuild"] == rebuilds[k], (k, st["rebuild"], rebuilds[k])
            assert st["rebuilds"] == sum(rebuilds[:k + 1])
        if kind == "refine":
            q, used = mark[2], mark[3]
            assert st["refine_done"] == (1 if q == used - 1 else 0), (k, q, used)
        if kind in ("after", "test") and k < n_iters - 1:
            assert st["done"] == 0, (kind, k)
        if kind == "after" and st["done"]:
            last = st
            break
        last = st
    assert last["done"] == 1
    assert last["status"] == status
    assert last["k"] == k_done
    assert last["ksp_total"] == ksp_total
    assert last["refine_steps"] == steps
