"""Train the learned warm start on the GPU and write its weights.

    python pismv0.7.3_b200/train_warm_start.py --cases 2000 --steps 4000 --out weights.npz

1. Training data: ``--cases`` seeded synthetic ice sheets at 401 x 401 (10 km over the
   4000 km domain of the 801 x 801 benchmark, so the 801^2 inputs subsampled by 2 are drawn
   from the same distribution), each solved by the FP64 Picard / BiCGStab + multigrid path
   (``learned.solve_config``) on one solver handle.
   ``--gen-seconds`` caps the generation time; the cases solved by then are used.
2. Training: Adam on random ``--crop``^2 crops (flips / transposes), weighted MSE on
   asinh(u / 10 m/yr) (weight 1 on ice, 0.2 off ice), with the network's own CUDA kernels.
3. Evaluation: the loss on held-out 401^2 seeds, and on the unseen 801^2 seed-0 benchmark
   sheet the Picard iterations and time of the fast solve from zero and from the learned
   guess (features at stride 2, the prediction interpolated back to 801^2).
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


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", type=int, default=2000)
    ap.add_argument("--val-cases", type=int, default=16)
    ap.add_argument("--gen-seconds", type=float, default=600.0)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--crop", type=int, default=128)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None)
    ap.add_argument("--report", default=None)
    ap.add_argument("--eval-size", type=int, default=801)
    args = ap.parse_args(argv)

    _package()
    sys.path.insert(0, REPO)
    import numpy as np
    import torch
    import bench
    from pism_b200 import learned as L
    from pism_b200.ssa import SSAFD

    def log(m):
        print(m, flush=True)

    dev = torch.device("cuda", 0)
    report = {"args": vars(args)}

    # 1. data (the generation loop stops starting new chunks after gen-seconds)
    t0 = time.perf_counter()
    seeds = list(range(args.cases))
    data, stats = [], []
    chunk = 32
    for start in range(0, len(seeds), chunk):
        if time.perf_counter() - t0 > args.gen_seconds:
            break
        d, s = L.generate(seeds[start:start + chunk])
        data += d
        stats += s
        log(f"generated {len(data)} cases in {time.perf_counter() - t0:.0f} s")
    gen_s = time.perf_counter() - t0
    val, _ = L.generate(list(range(1_000_000, 1_000_000 + args.val_cases)))
    report["generation"] = {"cases": len(data), "seconds": gen_s,
                            "mean_picard": float(np.mean([s["picard"] for s in stats])),
                            "unconverged": int(sum(1 for s in stats if not s["converged"]))}
    log(json.dumps(report["generation"]))

    # 2. training
    net = L.UNet(args.batch, args.crop, args.crop, seed=args.seed)
    evalnet = L.UNet(1, 408, 408, params=net.get_params())
    report["val_loss_init"] = L.evaluate(evalnet, val)
    t1 = time.perf_counter()
    hist = L.train(net, data, steps=args.steps, batch=args.batch, crop=args.crop, lr=args.lr, seed=args.seed, log=log)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t1
    evalnet.set_params(net.get_params())
    report["training"] = {"steps": args.steps, "seconds": train_s, "ms_per_step": 1e3 * train_s / args.steps,
                          "loss_first100": float(np.mean(hist[:100])), "loss_last100": float(np.mean(hist[-100:]))}
    report["val_loss"] = L.evaluate(evalnet, val)
    report["train_loss_whole_images"] = L.evaluate(evalnet, data[:args.val_cases])
    log(json.dumps(report["training"]) + f" val {report['val_loss']:.5f} (init {report['val_loss_init']:.5f})")
    if args.out:
        net.save(args.out, cases=len(data), steps=args.steps, val_loss=report["val_loss"])

    # 3. the unseen benchmark sheet
    M = args.eval_size
    g, c_plain, f, _ = bench.build_case(M)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    names = ("thickness", "surface", "bed", "mask", "tauc", "melange")
    dfields = {k: torch.tensor(f[k], dtype=torch.float64, device=dev) for k in names}
    hh, ww = L.image_shape(M, M, 2)
    enet = L.UNet(1, hh, ww, params=net.get_params())
    enet.set_stream(stream.cuda_stream)

    def run(cfg, learned):
        s = SSAFD(g, cfg)
        s.set_stream(stream.cuda_stream)
        s.set_inputs(**dfields)
        out = torch.empty((M, M, 2), dtype=torch.float64, device=dev)
        for _ in range(2):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            if learned:
                L.learned_guess(s, enet, 2)
            else:
                s.set_initial_guess(torch.zeros_like(out))
            guess = s.velocity(out=torch.empty_like(out))
            s.solve(out=out)
            e1.record(stream)
            torch.cuda.synchronize()
        st = s.stats()
        s.close()
        return out, guess, e0.elapsed_time(e1), st

    ref, _, t_plain, st_plain = run(c_plain, False)
    fast = bench.fast_config(c_plain)
    u0, _, t0f, st0 = run(fast, False)
    u1, guess, t1f, st1 = run(fast, True)
    n = float(ref.norm())
    report["benchmark_801"] = {
        "plain_ms": t_plain, "plain_picard": st_plain["picard_iterations"],
        "fast_zero_ms": t0f, "fast_zero_picard": st0["picard_iterations"],
        "fast_learned_ms": t1f, "fast_learned_picard": st1["picard_iterations"],
        "guess_rel_l2_vs_plain": float((guess - ref).norm()) / n,
        "fast_zero_rel_l2_vs_plain": float((u0 - ref).norm()) / n,
        "fast_learned_rel_l2_vs_plain": float((u1 - ref).norm()) / n,
    }
    log(json.dumps(report["benchmark_801"]))
    if args.report:
        with open(args.report, "w") as fh:
            json.dump(report, fh, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
