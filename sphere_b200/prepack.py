"""Creates the settled packing of the dense-shear workload on the GPU:
    python -m sphere_b200.prepack [--n 100000] [--seed 1] [--out packing.bin]
    python -m sphere_b200.prepack --pack packing.bin   (writes the packaged fixture)

The packing is input preparation for the benchmark and the tests: damped
settling on the GPU engine (configs.settle_packing).  The 100,000-sphere
packing of seed 1 ships with the package (sphere_b200/data, written by
--pack from a settled .bin), so the benchmark and its CPU reference arm read
the same input without settling anything; other sizes are settled on demand
and cached under $SPHB_CACHE (default: a folder in the system's temporary
directory)."""
import argparse
import sys

from . import binfile, configs


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=100000)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=None, help="also write the settled packing as a .bin file")
    ap.add_argument("--pack", default=None,
                    help="store this settled .bin as the packaged fixture and exit")
    a = ap.parse_args(argv)
    if a.pack:
        path = configs.pack_fixture(binfile.read_bin(a.pack), a.seed)
        print(f"fixture written: {path}", flush=True)
        return
    base = configs.settled_packing(n=a.n, seed=a.seed, packaged=False,
                                   log=lambda m: print(m, file=sys.stderr, flush=True))
    if a.out:
        binfile.write_bin(base, a.out)
    print(f"packing ready: {base.np} particles, grid {list(base.num)}", flush=True)


if __name__ == "__main__":
    main()
