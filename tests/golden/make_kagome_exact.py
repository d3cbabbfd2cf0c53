"""Extended-precision equal-time Green's functions for the kagome golden case.

The kagome case (N = 48, L = 40, U = 6, beta = 4) is the least well
conditioned of the golden cases: the FP64 stabilised G of the oracle and of
the GPU engine agree there only to a few 1e-9.  This script decides which
side carries that error.  It runs the oracle for five sweeps (the fields are
bit-exact between oracle, reference build and engine), then evaluates

    G_s = (I + B_{L-1} ... B_0)^-1,   B_l = exp_K_s diag(exp_lambda[hs_l ^ s])

with 50 significant digits (mpmath), taking the FP64 exp_K and exp_lambda
of the sim file as exact inputs -- the same inputs both FP64 computations
start from.  It writes tests/golden/kat_kagome/g_exact_5.npz: the fields
after five sweeps and G_up, G_dn rounded to FP64.

Runs on the CPU in about a minute:  python tests/golden/make_kagome_exact.py
"""
import os
import shutil
import sys
import tempfile

import mpmath as mp
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "dqmc-dev_b200"))

from oracle_ctl import Sim  # noqa: E402

CASE = os.path.join(HERE, "kat_kagome")
SWEEPS = 5
DIGITS = 50


def exact_g(expK, el, hs, spin):
    """(I + B_{L-1} ... B_0)^-1 in DIGITS-digit arithmetic, FP64 result"""
    L, N = hs.shape
    K = mp.matrix(N, N)
    for i in range(N):
        for j in range(N):
            K[i, j] = mp.mpf(float(expK[i, j]))
    P = mp.eye(N)
    for l in range(L):
        d = [mp.mpf(float(el[i + N * (int(hs[l, i]) ^ spin)])) for i in range(N)]
        for j in range(N):          # P <- diag(d) P
            for i in range(N):
                P[i, j] *= d[i]
        P = K * P                   # P <- exp_K P
    G = mp.inverse(mp.eye(N) + P)
    return np.array([[float(G[i, j]) for j in range(N)] for i in range(N)])


def main():
    mp.mp.dps = DIGITS
    tmp = tempfile.mkdtemp()
    try:
        for f in ("sim_0.h5", "sim.h5.params"):
            shutil.copy(os.path.join(CASE, f), tmp)
        o = Sim(os.path.join(tmp, "sim_0.h5"))
        gu_o, gd_o, _ = o.run(stop_sweep=SWEEPS)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    N, L = o.N, o.L
    hs = o.hs.reshape(L, N).copy()
    el = o.a["exp_lambda"]
    gu = exact_g(o.a["exp_Ku"].reshape(N, N).T, el, hs, 0)
    gd = exact_g(o.a["exp_Kd"].reshape(N, N).T, el, hs, 1)
    out = os.path.join(CASE, f"g_exact_{SWEEPS}.npz")
    np.savez_compressed(out, hs=hs, gu=gu, gd=gd, sweeps=SWEEPS, digits=DIGITS)
    print(f"wrote {out}")
    print(f"oracle max |G - G_exact|: up {np.max(np.abs(gu_o - gu)):.3e}, "
          f"down {np.max(np.abs(gd_o - gd)):.3e}")


if __name__ == "__main__":
    main()
