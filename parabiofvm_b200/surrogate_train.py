"""Train the surrogate of the standard 128^3 x 4 microenvironment and save its parameters.

    python -m parabiofvm_b200.surrogate_train --out surrogate_128x4.npz [--pairs 2000] [--minutes 10]

The data set is 2,000 pairs from the plain GPU solver (fields of 8 Gaussian bumps per substrate,
10,000-100,000 uniformly placed agents, the field 16 plain steps later), regenerated from their
seeds every epoch (PairGenerator.fill with a pair index).  Adam at learning rate 1e-3 on batches
of 4 pairs, all in this library's kernels.  After every epoch the network is evaluated on 16 pairs
outside the training set; training stops after --epochs epochs, once an epoch ends past
--minutes, or once the held-out error has not improved by 1 % for --patience epochs (the
plateau).  The output holds the parameters of the epoch with the lowest held-out error and a JSON
record: the environment, the recipe and the per-epoch curve.
"""

from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", required=True, help="output .npz (parameters and training record)")
    ap.add_argument("--pairs", type=int, default=2000)
    ap.add_argument("--held-out", type=int, default=16)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--learning-rate", type=float, default=1e-3)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--minutes", type=float, default=10.0)
    ap.add_argument("--patience", type=int, default=3)
    ap.add_argument("--seed", type=int, default=7, help="initial weights")
    ap.add_argument("--data-seed", type=int, default=11, help="the data set's pairs")
    args = ap.parse_args(argv)

    import torch

    from . import surrogate as su

    torch.cuda.set_device(0)
    env = su.standard_environment()
    net = su.Surrogate(env.grid, env.S, max_batch=args.batch, seed=args.seed)
    gen = su.PairGenerator(env, seed=args.data_seed)
    held_out = list(range(args.pairs, args.pairs + args.held_out))

    t0 = time.perf_counter()
    before = su.evaluate(net, gen, held_out)
    curve = [{"epoch": 0, "steps": 0, "held_out_rel_l2": before[0], "held_out_rel_l2_without_net": before[1],
              "seconds": 0.0}]
    print(json.dumps(curve[-1]), file=sys.stderr, flush=True)
    best = (before[0], net.save(), 0)
    order_rng = np.random.default_rng(args.seed)
    stale = 0
    for epoch in range(1, args.epochs + 1):
        ep = su.train_on_pairs(net, gen, args.pairs, 1, batch=args.batch, learning_rate=args.learning_rate,
                               held_out=held_out, seed=int(order_rng.integers(1 << 31)))[0]
        ep["epoch"] = epoch
        ep["steps"] = epoch * (args.pairs // args.batch)
        ep["seconds"] = time.perf_counter() - t0
        curve.append(ep)
        print(json.dumps(ep), file=sys.stderr, flush=True)
        if ep["held_out_rel_l2"] < best[0] * 0.99:
            best = (ep["held_out_rel_l2"], net.save(), epoch)
            stale = 0
        else:
            stale += 1
            if ep["held_out_rel_l2"] < best[0]:
                best = (ep["held_out_rel_l2"], net.save(), epoch)
        if stale >= args.patience or ep["seconds"] > args.minutes * 60:
            break

    record = {
        "environment": {"grid": list(env.grid), "dx": env.dx, "time_step": env.time_step,
                        "diffusion_coefficients": env.diffusion_coefficients, "decay_rates": env.decay_rates},
        "recipe": {"pairs": args.pairs, "batch": args.batch, "optimizer": "Adam", "learning_rate": args.learning_rate,
                   "init_seed": args.seed, "data_seed": args.data_seed, "held_out_pairs": held_out,
                   "agents_per_pair": list(gen.agents), "macro_steps": su.MACRO_STEPS},
        "best_epoch": best[2],
        "held_out_rel_l2": best[0],
        "held_out_rel_l2_without_net": before[1],
        "curve": curve,
    }
    np.savez_compressed(args.out, parameters=best[1], record=json.dumps(record))
    print(json.dumps({"out": args.out, "best_epoch": best[2], "held_out_rel_l2": best[0],
                      "held_out_rel_l2_without_net": before[1], "epochs": len(curve) - 1,
                      "seconds": time.perf_counter() - t0}), flush=True)
    gen.close()
    net.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
