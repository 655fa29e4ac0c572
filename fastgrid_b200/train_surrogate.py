"""Train the e-map surrogate's corrector network on the GPU and save its weights.

    python -m fastgrid_b200.train_surrogate [--receptors 200] [--epochs 10] [--out FILE] [--report FILE]

The receptors are seeded synthetic globules (5,000-30,000 atoms by default)
whose e-maps the direct kernel computes; the forward and backward passes and
the Adam updates run in the library's own CUDA kernels (ag_surrogate_train).
Prints one JSON line with the timings and the loss per epoch, and writes it
(with the SHA-256 of the weights file and the GPU's name) to the report file:
the shipped fastgrid_b200/surrogate_weights.bin comes with its report,
fastgrid_b200/surrogate_weights.json.
"""
import argparse
import hashlib
import json
import os

import fastgrid_b200 as fg


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--receptors", type=int, default=200)
    ap.add_argument("--min-atoms", type=int, default=5000)
    ap.add_argument("--max-atoms", type=int, default=30000)
    ap.add_argument("--points", type=int, default=161)
    ap.add_argument("--spacing", type=float, default=0.375)
    ap.add_argument("--epochs", type=int, default=10)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=fg.DEFAULT_WEIGHTS)
    ap.add_argument("--report", default=None, help="JSON report (default: the weights file with .json)")
    a = ap.parse_args(argv)
    ctx = fg.Context(0)
    rep = ctx.surrogate_train(n_receptors=a.receptors, min_atoms=a.min_atoms, max_atoms=a.max_atoms,
                              points=a.points, spacing=a.spacing, epochs=a.epochs, lr=a.lr, seed=a.seed)
    ctx.surrogate_save(a.out)
    ctx.close()
    rep.update(receptors=a.receptors, atoms=[a.min_atoms, a.max_atoms], points=a.points, spacing=a.spacing,
               epochs=a.epochs, lr=a.lr, seed=a.seed, weights=os.path.basename(a.out),
               weights_sha256=hashlib.sha256(open(a.out, "rb").read()).hexdigest(),
               command="python -m fastgrid_b200.train_surrogate " + " ".join(
                   f"--{k} {v}" for k, v in (("receptors", a.receptors), ("min-atoms", a.min_atoms),
                                             ("max-atoms", a.max_atoms), ("points", a.points),
                                             ("spacing", a.spacing), ("epochs", a.epochs), ("lr", a.lr),
                                             ("seed", a.seed))))
    try:
        import torch
        rep["gpu"] = torch.cuda.get_device_name(0)
    except Exception:
        pass
    line = json.dumps(rep)
    print(line)
    with open(a.report or os.path.splitext(a.out)[0] + ".json", "w") as f:
        f.write(json.dumps(rep, indent=1) + "\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
