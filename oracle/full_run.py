"""One complete run of the native CPU restatement of SSAFD's Picard loop on the bench's
synthetic sheet, and the fit of its per-Picard set-up cost: the numbers behind the CPU
baseline's cost model in bench.py (CPU_FULL_RUN_801).

    python oracle/full_run.py --size 801 --threads 8 --picard-rtol 1e-6 --out run.json

Oracle infrastructure (timing the CPU restatement, never the product): it runs
oracle/ssafd_cpu.cc through oracle.ssafd_oracle.picard_native from a zero guess with KSP rtol
1e-8, as the reference's default KSP would, and prints one JSON line with the counts and the fit
`t_k = a + b its_k` (least squares with 4-MAD outlier rejection) of the Picard iterations'
seconds t_k against their GMRES iterations its_k.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def fit_setup(seconds, its):
    """(a, b, kept) of t = a + b its, refitted without residuals beyond 4 scaled MADs"""
    t = np.asarray(seconds, float)
    A = np.vstack([np.ones(len(its)), np.asarray(its, float)]).T
    keep = np.ones(len(t), bool)
    coef = np.zeros(2)
    for _ in range(10):
        coef = np.linalg.lstsq(A[keep], t[keep], rcond=None)[0]
        r = t - A @ coef
        mad = np.median(np.abs(r[keep] - np.median(r[keep])))
        new = np.abs(r) < 4 * 1.4826 * mad if mad > 0 else keep
        if (new == keep).all():
            break
        keep = new
    return float(coef[0]), float(coef[1]), int(keep.sum())


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=801)
    ap.add_argument("--threads", type=int, default=8)
    ap.add_argument("--picard-rtol", type=float, default=1e-6)
    ap.add_argument("--max-iterations", type=int, default=5000)
    ap.add_argument("--out", default=None, help="also write the per-iteration record as JSON here")
    args = ap.parse_args(argv)
    sys.path.insert(0, REPO)
    import bench
    from oracle import ssafd_oracle as O
    g, c, f, _ = bench.build_case(args.size)
    G, Cc, I = O.from_case(g, c, f)
    t0 = time.perf_counter()
    o = O.SSAFDOracle(G, Cc, I)
    o.prepare()
    t1 = time.perf_counter()
    _, info = O.picard_native(G, Cc, I, o.hardness, o.b, np.zeros((args.size, args.size, 2)), Cc.epsilon_ssa,
                              nranks=args.threads, nthreads=args.threads, ksp_rtol=1e-8,
                              max_iterations=args.max_iterations, picard_rtol=args.picard_rtol)
    total = time.perf_counter() - t1
    per = [a + b + d for a, b, d in zip(info["t_nuH"], info["t_assemble"], info["t_ksp"])]
    its = [int(k) for k in info["ksp_iterations"]]
    a, b, kept = fit_setup(per, its)
    change = np.asarray(info["rel_change"])
    summary = {"size": args.size, "threads": args.threads, "status": info["status"], "prepare_s": t1 - t0,
               "total_s": total, "picard_iterations": len(its), "ksp_iterations": sum(its),
               "first_ksp_iterations": its[:3], "fit": {"a_s": a, "b_s": b, "setup_iterations": a / b, "kept": kept}}
    for tol in (1e-4, 1e-6):
        hit = np.nonzero(change <= tol)[0]
        if len(hit):
            k = int(hit[0]) + 1
            summary[f"to_{tol:g}"] = {"picard_iterations": k, "ksp_iterations": sum(its[:k]), "seconds": sum(per[:k])}
    print(json.dumps(summary))
    if args.out:
        with open(args.out, "w") as fh:
            json.dump({**summary, "seconds": per, "its": its, "rel_change": list(map(float, change))}, fh)
    return 0


if __name__ == "__main__":
    sys.exit(main())
