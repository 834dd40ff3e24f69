"""A self-contained solve for profilers (ncu): one instance of a chosen size,
one solve with an iteration cap, result printed.

    python -m reformulation_b200.profile_case praq --n 100000 --m 1000000 --max-iter 64
    python -m reformulation_b200.profile_case praq --n 2000000 --m 20000000 --max-iter 48

The PRAQ instance is `qubo_uniform_edges` (uniform distinct pairs, integer
weights); the size is chosen so that the captured kernels' inputs are larger
than L2 (126 MB) when DRAM figures are wanted, and a few GB at most.
"""

from __future__ import annotations

import argparse
import time


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("path", choices=("praq", "pria"))
    ap.add_argument("--n", type=int, default=100_000)
    ap.add_argument("--m", type=int, default=1_000_000)
    ap.add_argument("--items", type=int, default=100)
    ap.add_argument("--periods", type=int, default=500)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--max-iter", type=int, default=64)
    ap.add_argument("--tol", type=float, default=1e-4)
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="mixed")
    args = ap.parse_args()
    if args.path == "praq":
        from . import praq
        from .instances import qubo_uniform_edges
        inst = qubo_uniform_edges(args.seed, args.n, args.m)
        lib = praq.Library()
        p = lib.parameters(tolerance=args.tol, max_iter=args.max_iter,
                           use_float32=int(args.precision == "mixed"))
        with praq.DeviceSolver(inst, p) as dev:
            t0 = time.perf_counter()
            st = dev.run()
            dt = time.perf_counter() - t0
            r = dev.result(want_x=False)
        print(f"praq n={args.n} m={args.m} status={st} iterations={r.iterations} "
              f"lower={r.lower:.10g} upper={r.upper:.10g} seconds={dt:.4f}")
        return 0 if st >= 0 else 1
    from . import pria
    from .instances import jrp_demand
    inst = jrp_demand(args.seed, args.items, args.periods)
    res = pria.solve_arrays(inst, tolerance=args.tol, max_iter=args.max_iter,
                            precision=args.precision)
    print(f"pria N={args.items} T={args.periods} iterations={res['iterations']} "
          f"lower={res['lower']:.10g} upper={res['upper']:.10g}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
