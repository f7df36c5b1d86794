"""Generates the golden fixtures of this directory by running the reference's own splatting
extension (built from the reference sources by ``oracle/build_ref.py`` into ``oracle/_ref``)
on a CUDA device, in float32 and in float64 (the reference dispatches both,
``PyOptix/kernel/photon_differentials.cu:124``, ``:233``).

    python tests/golden/make_golden.py [--out DIR]

Each case is a seeded photon set (from ``shapefromcaustics_b200.synthetic``, drawn on the
CPU) plus an upstream gradient; the fixture stores the float32 inputs and the reference's
forward image and gradients in both precisions. ``tests/test_golden.py`` pins the CPU oracle
on them. Cases cover the uniform/cluster workload, several channels including out-of-range
ones, photons on and off the image edges, a tiny image (the reference's ellipse test), a
photon exactly on a pixel corner (the reference's 0/0 in the backward) and a truncating
max_pixel_radius.
"""
import argparse
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from shapefromcaustics_b200 import synthetic as S  # noqa: E402


def cases():
    out = {}
    ph = S.uniform_cluster_photons(3000, 96, 96, seed=21, sigma=6.0)
    out["uniform_cluster_96"] = (ph, (1, 96, 96), 20)

    n = 2500
    E, X, M, C, R = S.uniform_cluster_photons(n, 48, 80, seed=22, s_range=(0.5, 6.0), sigma=5.0)
    # channels 3 and 4 lie outside C = 3 and are skipped by the reference (:75); negative
    # channels are left out: the reference indexes memory before its output with them
    C = torch.randint(0, 5, (1, n), generator=torch.Generator().manual_seed(22))
    out["channels_ragged_48x80"] = ((E, X, M, C, R), (3, 48, 80), 20)

    g = torch.Generator().manual_seed(23)
    n = 2000
    pos = torch.rand((2, n), generator=g, dtype=torch.float64) * 80 - 8
    th = torch.rand(n, generator=g, dtype=torch.float64) * np.pi
    s1 = 0.5 + torch.rand(n, generator=g, dtype=torch.float64) * 5
    s2 = 0.5 + torch.rand(n, generator=g, dtype=torch.float64) * 5
    e = torch.rand(n, generator=g, dtype=torch.float64) - 0.2
    out["edges_64"] = (S.photons_from_pixels(pos, th, s1, s2, e, 64, 64), (1, 64, 64), 20)

    out["tiny_8"] = (S.uniform_cluster_photons(300, 8, 8, seed=24, s_range=(2.0, 20.0), sigma=2.0),
                     (1, 8, 8), 20)

    # one photon exactly on a pixel corner, among others
    E, X, M, C, R = S.uniform_cluster_photons(200, 32, 32, seed=25)
    X[0, 0] = 2 * 10 / 32 - 1
    X[1, 0] = 2 * 12 / 32 - 1
    out["corner_32"] = ((E, X, M, C, R), (1, 32, 32), 20)

    out["mpr2_64"] = (S.uniform_cluster_photons(1500, 64, 64, seed=26, s_range=(1.0, 8.0)),
                      (1, 64, 64), 2)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    a = ap.parse_args()
    from oracle import build_ref
    ref = build_ref.load_module()
    dev = torch.device("cuda:0")
    os.makedirs(a.out, exist_ok=True)
    for name, ((E, X, M, C, R), shape, mpr) in cases().items():
        G = S.upstream_grad(shape, seed=sum(map(ord, name)))
        rec = dict(E=E.numpy(), X=X.numpy(), M=M.numpy(), C=C.numpy(), R=R.numpy(),
                   G=G.numpy(), shape=np.array(shape), mpr=np.array(mpr))
        for tag, dt in (("f32", torch.float32), ("f64", torch.float64)):
            args = [t.to(dev, dt).contiguous() for t in (E, X, M)] + [C.to(dev)] + [R.to(dev, dt)]
            img = ref.pds_forward(*args, list(shape), mpr)[0]
            gE, gX, gM = ref.pds_backward(G.to(dev, dt).contiguous(), *args, mpr)
            torch.cuda.synchronize()
            rec[f"img_{tag}"] = img.cpu().numpy()
            rec[f"gE_{tag}"] = gE.cpu().numpy()
            rec[f"gX_{tag}"] = gX.cpu().numpy()
            rec[f"gM_{tag}"] = gM.cpu().numpy()
        np.savez_compressed(os.path.join(a.out, f"{name}.npz"), **rec)
        print("wrote", name)


if __name__ == "__main__":
    main()
