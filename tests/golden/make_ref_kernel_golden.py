"""Run the reference's own CUDA sort / resampling / ring-exchange kernels
(oracle/_ref/libref_kernels.so, built by oracle/build_ref_kernels.sh) on the
committed golden inputs and store their outputs in ref_kernels.npz beside this
script.  Needs a GPU (run it on one; the library travels with the repository
snapshot).  The CPU tests then check the oracle's golden outputs against them."""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent / "oracle"))
import ref_kernels as R  # noqa: E402


def main():
    g = np.load(HERE / "golden.npz")
    out = {}
    for m in (32, 64, 256, 512):
        k, p = R.block_sort(g["sort_in_%d" % m], m)
        out["sort_key_%d" % m], out["sort_idx_%d" % m] = k, p
        out["res_ref_%d" % m] = R.resampling(g["res_w_%d" % m], g["res_uref_%d" % m], m)
    # ring routing: 8 sub-filters of 32, t = 3 (slot sources of the replaced slots)
    N, m, t = 8, 32, 3
    keys = -np.sort(-np.random.default_rng(7).standard_normal((N, m)).astype(np.float32), axis=1).reshape(-1)
    _, src = R.exchange_ring(keys, m, t)
    out["exch_src_1_8_32_3"] = np.ascontiguousarray(src.reshape(N, m)[:, m - t:])
    np.savez_compressed(HERE / "ref_kernels.npz", **out)
    print("wrote", HERE / "ref_kernels.npz", sorted(out))


if __name__ == "__main__":
    main()
