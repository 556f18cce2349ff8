"""Train the learned preconditioner correction of flexible GMRES on the GPU and write its weights.

    python pismv0.7.3_b200/train_learned_pc.py --cases 1000 --steps 10000 --out weights.npz

1. Training data (``learned.generate_pc``): seeded synthetic sheets at 401 x 401 (10 km, the
   distributions of the warm start's training set), each solved to a Picard tolerance of 1e-2
   by the FP64 FGMRES + multigrid path; per sheet a few random vectors v, the residual the
   multigrid cycle leaves, r = v - A M^-1 v, and the error e = A^-1 r that removes it.
2. Training: Adam on random ``--crop``^2 crops (flips / transposes: the residual channels and
   the error change sign and swap as the driving stress and the velocity do for the warm
   start), weighted MSE between the network's output and e / rho, with the network's own
   CUDA kernels.
3. Evaluation (``evaluate_gain``): on sheets outside the training seeds (401^2 at stride 1 and
   the 801^2 benchmark sheet at stride 2), FGMRES(30) + multigrid to relative residual 1e-8
   from zero at a Picard iterate, with and without the correction: iterations and time.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def _package():
    if "pism_b200" not in sys.modules:
        spec = importlib.util.spec_from_file_location("pism_b200", os.path.join(HERE, "__init__.py"),
                                                      submodule_search_locations=[HERE])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["pism_b200"] = mod
        spec.loader.exec_module(mod)
    return sys.modules["pism_b200"]


def evaluate_gain(net, g, c, f, stride, device=0, picard_rtol=1e-2, rtol=1e-8, reps=2):
    """FGMRES(30) + multigrid from zero at the Picard iterate of picard_rtol: (iterations,
    ms) without and with the learned correction"""
    import torch
    from pism_b200 import learned as L
    from pism_b200.ssa import SSAFD
    dev = torch.device("cuda", device)
    M = (g.Mx, g.My)
    s = SSAFD(g, L.pc_config(c).copy(ssafd_relative_convergence=picard_rtol, ksp_rtol=1e-8), device=device)
    try:
        s.set_inputs(**{k: f[k] for k in ("thickness", "surface", "bed", "mask", "tauc", "melange")})
        s.set_initial_guess(torch.zeros((*M, 2), dtype=torch.float64, device=dev))
        s.solve(out=torch.empty((*M, 2), dtype=torch.float64, device=dev))
        s.set_config(L.pc_config(c).copy(ksp_rtol=rtol))
        out = {}
        for name, attach in (("multigrid", False), ("multigrid+learned", True)):
            L.set_learned_pc(s, net if attach else None, stride)
            ts = []
            for _ in range(reps + 1):
                x = torch.zeros((*M, 2), dtype=torch.float64, device=dev)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                its, res = s.linear_solve(x)
                e1.record()
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
            out[name] = {"iterations": its, "residual": res, "ms": float(sum(ts[1:]) / reps)}
        L.set_learned_pc(s, None, stride)
        return out
    finally:
        s.close()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", type=int, default=1000)
    ap.add_argument("--samples", type=int, default=4)
    ap.add_argument("--val-cases", type=int, default=16)
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--crop", type=int, default=128)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--gen-seconds", type=float, default=900.0)
    ap.add_argument("--out", default=None)
    ap.add_argument("--report", default=None)
    args = ap.parse_args(argv)

    _package()
    sys.path.insert(0, REPO)
    import numpy as np
    import torch
    import bench
    from pism_b200 import learned as L

    def log(m):
        print(m, flush=True)

    report = {"args": vars(args)}
    t0 = time.perf_counter()
    data = []
    seeds = list(range(args.cases))
    for start in range(0, len(seeds), 32):
        if time.perf_counter() - t0 > args.gen_seconds:
            break
        data += L.generate_pc(seeds[start:start + 32], samples=args.samples)
        log(f"generated {len(data)} pairs in {time.perf_counter() - t0:.0f} s")
    report["generation"] = {"pairs": len(data), "sheets": len(data) // args.samples,
                            "seconds": time.perf_counter() - t0}
    val = L.generate_pc(list(range(1_000_000, 1_000_000 + args.val_cases)), samples=2)

    net = L.UNet(args.batch, args.crop, args.crop, seed=args.seed)
    evalnet = L.UNet(1, 408, 408, params=net.get_params())
    report["val_loss_init"] = L.evaluate(evalnet, val)
    t1 = time.perf_counter()
    # the warm start's augmentation applies as it is: the residual channels 6, 7 and the error
    # change sign and swap like the driving stress and the velocity do
    hist = L.train(net, data, steps=args.steps, batch=args.batch, crop=args.crop, lr=args.lr, seed=args.seed,
                   log=log)
    torch.cuda.synchronize()
    report["training"] = {"steps": args.steps, "seconds": time.perf_counter() - t1,
                          "loss_first100": float(np.mean(hist[:100])), "loss_last100": float(np.mean(hist[-100:]))}
    evalnet.set_params(net.get_params())
    report["val_loss"] = L.evaluate(evalnet, val)
    log(json.dumps({k: report[k] for k in ("val_loss_init", "val_loss", "training")}))
    if args.out:
        evalnet.save(args.out, val_loss=report["val_loss"])

    # the gain on unseen sheets: 401^2 at stride 1, the 801^2 benchmark sheet at stride 2
    gains = []
    for seed in (2_000_001, 2_000_002):
        g, c, f, _ = L.training_case(seed, 401)
        gains.append({"sheet": f"401^2 seed {seed}", **evaluate_gain(evalnet, g, c, f, 1)})
        log(json.dumps(gains[-1]))
    big = L.UNet(1, 408, 408, params=net.get_params())
    g, c, f, _ = bench.build_case(801)
    gains.append({"sheet": "801^2 benchmark sheet (seed 0), stride 2", **evaluate_gain(big, g, c, f, 2)})
    log(json.dumps(gains[-1]))
    report["gain"] = gains
    if args.report:
        with open(args.report, "w") as fh:
            json.dump(report, fh, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
