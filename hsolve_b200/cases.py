"""Timing cases of the shift-invert path on the synthetic Yee/FIT pencils, for profiling runs.

    python -m hsolve_b200.cases factor [--case box1e5] [--shift 120] [--repeat 3]
    python -m hsolve_b200.cases solve  [--case box1e5] [--shift 120] [--nrhs 8] [--repeat 5]
    python -m hsolve_b200.cases eigs   [--case box1e5] [--repeat 4]

`factor` analyzes K = A - shift B once and factorizes it `repeat` times; `solve` factorizes once and
runs `repeat` in-place solves of `nrhs` device-resident right-hand sides; `eigs` runs the certified
solve of the case's target through a session `repeat` times. Each prints its wall times (and, for
`eigs`, the phase split of the solve report and the library's kernel launches before and during each
solve, which locate one solve in a profiler's launch list). The cases are the workloads of bench.py: box1e5 is
the PEC box 44 x 34 x 26 (lengths 1 x 0.75 x 0.55, generalized form, n = 109,744, all eigenvalues in
[40, 200]); cube20 is the PEC cube 20^3 (standard form, n = 21,660, 10 nearest to 25); cube70 is the
PEC cube 70^3 (n = 999,810, 21 nearest to 1071.43, between two exact levels); nedelec1e5 is the PEC
box 2 x 1 x 0.5 on 50 x 25 x 13 cells of six tetrahedra with lowest-order Nedelec elements
(consistent, non-diagonal mass; n = 107,163), all eigenvalues in [40, 200].
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from .gen import nedelec, yee


def _yee(box, form):
    a, b = yee.pencil(box, form)
    return a, (b if form == "generalized" else None)


CASES = {
    "box1e5": (lambda: _yee(yee.BOX_1E5, "generalized"), dict(lower=40.0, upper=200.0)),
    "cube20": (lambda: _yee(yee.CUBE20, "standard"), dict(sigma=25.0, k=10)),
    # PEC cube 70^3, n = 999,810: 21 nearest to a shift midway between two exact levels
    "cube70": (lambda: _yee(yee.Box((70, 70, 70)), "standard"), dict(sigma=1071.4257927949998, k=21)),
    "nedelec1e5": (lambda: nedelec.pencil(nedelec.BOX_2x1x05_1E5), dict(lower=40.0, upper=200.0)),
}


def _pencil(case):
    make, target = CASES[case]
    a, b = make()
    return a, b, target


def factor(case: str, shift: float, repeat: int) -> None:
    from ._native import Factorization

    a, b, _ = _pencil(case)
    f = Factorization(device=0)
    f.analyze(a, b, 1.0, -shift)
    for _ in range(repeat):
        t = time.perf_counter()
        ok = f.factorize(1.0, -shift)
        dt = time.perf_counter() - t
        print(f"factorize {1e3 * dt:.2f} ms valid={ok} {f.inertia()}", flush=True)


def solve(case: str, shift: float, nrhs: int, repeat: int) -> None:
    import torch

    from ._native import Factorization

    a, b, _ = _pencil(case)
    n = a.shape[0]
    f = Factorization(device=0)
    f.analyze(a, b, 1.0, -shift)
    assert f.factorize(1.0, -shift)
    rhs = np.random.default_rng(0).standard_normal((n, nrhs))
    dev = torch.from_numpy(np.ascontiguousarray(rhs.T)).cuda()
    x = None
    for _ in range(repeat):
        x = dev.clone()
        torch.cuda.synchronize()
        t = time.perf_counter()
        f.solve_device(x.data_ptr(), nrhs, n)
        torch.cuda.synchronize()
        print(f"solve {1e3 * (time.perf_counter() - t):.3f} ms ({nrhs} right-hand sides)", flush=True)
    import scipy.sparse as sp

    k = (a - shift * (b if b is not None else sp.identity(n))).tocsr()
    xs = x.cpu().numpy().T
    r = k @ xs - rhs
    print(f"backward error {np.abs(r).max() / (abs(k).sum(axis=0).max() * np.abs(xs).max()):.2e}")


def eigs(case: str, repeat: int) -> None:
    from ._native import kernel_launches
    from .api import Session

    a, b, target = _pencil(case)
    s = Session(a, b)
    for _ in range(repeat):
        l0 = kernel_launches()
        t = time.perf_counter()
        r = s.solve(**target)
        dt = time.perf_counter() - t
        rp = r.report
        print(f"solve {dt:.3f} s launches_before={l0} launches={kernel_launches() - l0} "
              f"success={r.success} eigenvalues={r.eigenvalues.size} "
              f"factor={rp['time_factor_s']:.4f} iterate={rp['time_iterate_s']:.4f} "
              f"certificate={rp['time_certificate_s']:.4f} verify={rp['time_verify_s']:.4f} "
              f"split={ {k: round(v, 4) for k, v in rp['iterate_split_s'].items()} }", flush=True)


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("what", choices=["factor", "solve", "eigs"])
    ap.add_argument("--case", default="box1e5", choices=sorted(CASES))
    ap.add_argument("--shift", type=float, default=120.0)
    ap.add_argument("--nrhs", type=int, default=8)
    ap.add_argument("--repeat", type=int, default=3)
    args = ap.parse_args(argv)
    if args.what == "factor":
        factor(args.case, args.shift, args.repeat)
    elif args.what == "solve":
        solve(args.case, args.shift, args.nrhs, args.repeat)
    else:
        eigs(args.case, args.repeat)


if __name__ == "__main__":
    main()
