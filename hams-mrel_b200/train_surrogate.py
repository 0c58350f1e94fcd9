"""Train the far-field Green-function surrogate on the GPU and store it.

    python hams-mrel_b200/train_surrogate.py [--steps 100000] [--samples 8000000] [--out PATH]

Samples come from the library's FINGREEN3D series (hams_surrogate_samples);
training runs in the library's own forward / backward / Adam kernels
(hams_surrogate_train).  The stored file is the raw float32 parameter vector
(hams_surrogate_param_count() values) that Context.set_surrogate takes; the
default output is the file the package ships and bench.py loads
(surrogate_w128x4.f32, trained with the defaults below: 16 M samples,
300 k steps of 16,384, peak learning rate 2e-3, seed 1; about 5 minutes on
one B200; held-out RMS error 3.2e-4, 3.8e-4, 4.3e-4 of the three outputs).
"""
import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import hams_b200 as hb  # noqa: E402

DEFAULT = os.path.join(HERE, "surrogate_w128x4.f32")


def load(path=DEFAULT):
    p = np.fromfile(path, dtype="<f4")
    if p.size != hb.surrogate_param_count():
        raise ValueError(f"{path}: {p.size} parameters, {hb.surrogate_param_count()} expected")
    return p


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--samples", type=int, default=16_000_000)
    ap.add_argument("--test", type=int, default=100_000)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--steps", type=int, default=300_000)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=DEFAULT)
    a = ap.parse_args()
    params, stats = hb.surrogate_train(n_train=a.samples, n_test=a.test, batch=a.batch, steps=a.steps, lr=a.lr,
                                       seed=a.seed)
    params.astype("<f4").tofile(a.out)
    print(json.dumps(dict(out=a.out, **stats)))


if __name__ == "__main__":
    main()
