"""Creates (or reuses) the cached settled packing of the dense-shear
workload:  python -m sphere_b200.prepack [--n 100000] [--seed 1]

The packing is input preparation for the benchmark and the tests; it is
made by damped settling on the GPU engine (configs.settle_packing) and
written to $SPHB_CACHE (default /tmp/sphere_b200_cache)."""
import argparse
import sys

from . import configs


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=100000)
    ap.add_argument("--seed", type=int, default=1)
    a = ap.parse_args(argv)
    d = configs.shear_benchmark(n=a.n, seed=a.seed,
                                log=lambda m: print(m, file=sys.stderr, flush=True))
    print(f"packing ready: {d.np} particles, grid {list(d.num)}", flush=True)


if __name__ == "__main__":
    main()
