"""Train the learned volume-fraction correction and write the packaged weights file.

    python cutcellmethods.jl_b200/train_correction.py [--out weights/mc_vf_correction.v1.bin]

The training set: 200 seeded bodies ``workloads.smooth_blob(seed)`` (smooth-min, k = 0.05, unions
of 4..12 spheres of radius U[0.05, 0.3] in the unit cube), seeds 1000..1199, body k on a grid of
(64 + 16 (k mod 13))^3 cells (64^3 .. 256^3), Float32 marching cubes; every cut cell is a sample
(corner phi / h, its plain fraction, the 8x sub-refined fraction). Training: the project's tcgen05
forward/backward kernels, Adam, 60000 steps of 32 x 128 samples, learning rate 2e-3 warmed up
over 10% and cosine-decayed, each sample under a random cube symmetry. Held-out evaluation: the
unseen bodies 5000 and 5001 at 512^3 (and 256^3), volume-fraction L1 error over the cut cells
against the 8x sub-refined labels, plain and learned. The training set is ordered by cell index
and training is deterministic, so a rerun on a B200 reproduces the file. Writes the weights and a
JSON summary (recipe, checksum, evaluation) beside them.
"""
from __future__ import annotations

import argparse
import importlib
import importlib.util
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))


def _package():
    name = "cutcell_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(HERE, "__init__.py"),
                                                  submodule_search_locations=[HERE])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


RECIPE = dict(bodies=200, seed0=1000, sizes=[64 + 16 * k for k in range(13)], steps=60000, tiles=32, lr=2e-3,
              train_seed=3, augment=True, init_seed=1, eval_seeds=[5000, 5001], eval_sizes=[256, 512], bound=0.05)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--out", default=os.path.join(HERE, "weights", "mc_vf_correction.v1.bin"))
    ap.add_argument("--steps", type=int, default=RECIPE["steps"])
    ap.add_argument("--bodies", type=int, default=RECIPE["bodies"])
    a = ap.parse_args(argv)
    import torch
    _package()
    L = importlib.import_module("cutcell_b200.learned")
    r = dict(RECIPE, steps=a.steps, bodies=a.bodies)
    t0 = time.time()
    data = L.training_set(range(r["seed0"], r["seed0"] + r["bodies"]), r["sizes"])
    torch.cuda.synchronize()
    t_data = time.time() - t0
    m = L.MLP(L.init_params(r["init_seed"]))
    t0 = time.time()
    loss = L.train_correction(m, data, steps=r["steps"], tiles=r["tiles"], lr=r["lr"], seed=r["train_seed"],
                              augment=r["augment"])
    torch.cuda.synchronize()
    t_train = time.time() - t0
    params = m.get_params()
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    L.save_weights(a.out, params)
    evals = [L.evaluate(m, s, n, bound=r["bound"]) for n in r["eval_sizes"] for s in r["eval_seeds"]]
    summary = dict(file=os.path.basename(a.out), version=L.WEIGHTS_VERSION, nparam=L.NPARAM,
                   fnv1a64=f"{L.fnv1a64(params.astype('<f4').tobytes()):016x}", recipe=r,
                   samples=int(data[0].shape[0]), data_seconds=round(t_data, 2), train_seconds=round(t_train, 2),
                   final_loss=loss, device=torch.cuda.get_device_name(), evaluation=evals)
    with open(os.path.splitext(a.out)[0] + ".json", "w") as fh:
        json.dump(summary, fh, indent=1)
    print(json.dumps(summary))


if __name__ == "__main__":
    main()
