"""Regenerates the golden fixtures of tests/golden/ from the FP64 oracle.

The reference (MATLAB, with its NUFFT and SARA primitives in un-vendored
submodules) cannot run here and ships no test vectors, so these fixtures pin
the oracle's own outputs on small seeded inputs: later changes to the oracle
(or to the GPU path checked against it) are caught as regressions.

Usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "faceted-hypersara_b200"))

from fhs_b200 import synth  # noqa: E402
from oracle import nufft, problem, wavelets  # noqa: E402
from oracle import solvers as so  # noqa: E402
from oracle.facets import FacetGeometry  # noqa: E402


def main():
    rng = np.random.default_rng(2024)
    # --- NUFFT: 16 x 12 image, 40 frequencies
    Ny, Nx = 16, 12
    op = nufft.NufftOperator(Ny, Nx)
    x = rng.standard_normal((Ny, Nx))
    om_y = rng.uniform(-np.pi, np.pi, 40)
    om_x = rng.uniform(-np.pi, np.pi, 40)
    G = op.G(om_y, om_x)
    np.savez_compressed(os.path.join(HERE, "nufft_16x12.npz"), x=x, om_y=om_y, om_x=om_x,
                        Fx=op.A(x), y=G @ op.A(x), sy=op.sy, sx=op.sx)
    # --- Daubechies filters db1..db8 (reconstruction low-pass, MATLAB orientation)
    filt = {f"db{p}": wavelets.daubechies_lo_r(p) for p in range(1, 9)}
    np.savez_compressed(os.path.join(HERE, "daubechies.npz"), **filt)
    # --- SARA analysis of a 13 x 10 x 2 cube
    xs = rng.standard_normal((2, 13, 10))
    np.savez_compressed(os.path.join(HERE, "sara_13x10x2.npz"), x=xs, coefs=wavelets.sara_analysis(xs))
    # --- 3 FHS iterations on a 24 x 24 x 2 problem, 2 x 2 facets
    data, xt, meta = problem.make_problem(24, 24, 2, 300, 2, seed=7, synth=synth)
    nu2 = so.operator_norm(data, 200, 1e-12)
    geom = FacetGeometry(24, 24, 2, 2, (3, 3))
    sig, sig_bar, *_ = so.compute_noise_level(24, 24, 2, np.ones(2), "fhs", geom, nu2)
    p = so.SolverParams(nu2=nu2, gamma=sig, gamma0=sig_bar, reweighting_sig=sig, reweighting_sig_bar=sig_bar,
                        pdfb_min_iter=10 ** 6, reweighting_flag=False)
    x3, _ = so.facet_hypersara(data, p, geom, max_iter=3)
    np.savez_compressed(os.path.join(HERE, "fhs_24x24x2_3iter.npz"), x3=x3, nu2=nu2, sig=sig, sig_bar=sig_bar,
                        om_y0=meta["om"][0][0], om_x0=meta["om"][0][1], om_y1=meta["om"][1][0],
                        om_x1=meta["om"][1][1], blocks=np.array(meta["blocks"]), sigma=np.array(meta["sigma"]),
                        y0=np.concatenate(data.y[0]), y1=np.concatenate(data.y[1]))
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
