"""Generate tests/golden/golden.npz.

* MTGP32 known-answer vectors come from the REFERENCE's own CPU generator
  (src/partfilt/cuda/mtgp/mtgp32-fast.c + mtgp32dc-param-11213.c from the
  Esthera tree, built by oracle/build_ref.sh into oracle/_ref/).
* Sort / scan / resampling / alias / routing vectors come from the CPU oracle
  (oracle/pf_oracle.c) on seeded inputs; the tests re-derive the small cases
  with independent pure-Python restatements.

Run here (where the reference tree exists): python tests/golden/make_golden.py
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import oracle as O  # noqa: E402

KAT_CASES = [(0, 1), (1, 1), (2, 1), (95, 0xF000000D), (119, 0xF000000D), (199, 0xF000000D), (0, 0xF000000D),
             (7, 12345)]
KAT_N = 1024


def main():
    if O.ref_lib() is None:
        raise SystemExit("oracle/_ref/libmtgp_ref.so missing: run oracle/build_ref.sh first")
    g = {}
    for set_, seed in KAT_CASES:
        g["kat_u32_%d_%d" % (set_, seed)] = O.ref_mtgp_stream(set_, seed, KAT_N, kind=0)
        g["kat_f32_%d_%d" % (set_, seed)] = O.ref_mtgp_stream(set_, seed, KAT_N, kind=1)
    # reference block layout, OpenCL deterministic seed, G = 96, two launches of 768 per stream
    G, per = 96, 768
    seed = 0xF000000D
    blk = []
    for call in range(2):
        out = np.zeros(G * per, np.uint32)
        for gg in range(G):
            s = O.ref_mtgp_stream(gg, (seed + gg + 1) & 0xFFFFFFFF, per * (call + 1), kind=1)
            out[gg * per:(gg + 1) * per] = s[call * per:(call + 1) * per]
        blk.append(out)
    g["blocks_G96_f32"] = np.concatenate(blk)
    # the reference CUDA kernel's hard-wired mask (oracle only: no runnable reference for it)
    g["cudamask_f32_0_1"] = O.mtgp_stream(0, 1, KAT_N, kind=1, mask=O.MASK_CUDA_REF)

    rng = np.random.default_rng(20240611)
    # bitonic sort: random keys, heavy ties, zeros (underflowed linear weights), negatives
    for m in (32, 64, 256, 512):
        keys = rng.standard_normal(4 * m).astype(np.float32)
        keys[m:2 * m] = np.round(keys[m:2 * m] * 2) / 2          # many ties
        keys[2 * m:3 * m] = 0.0
        keys[2 * m:2 * m + 5] = [1.0, 0.5, 1.0, 0.25, 1.0]      # mostly-zero sub-filter
        keys[3 * m:] = -np.abs(keys[3 * m:]) * 50                # log-weights
        sk, si = O.bitonic_sort(keys, m)
        g["sort_in_%d" % m], g["sort_key_%d" % m], g["sort_idx_%d" % m] = keys, sk, si
    # resamplers on linear weights
    for m in (32, 64, 256, 512):
        w = rng.exponential(1.0, 4 * m).astype(np.float32)
        w[m:2 * m] = (rng.random(m) < 0.05).astype(np.float32) * rng.random(m).astype(np.float32)
        w[2 * m:3 * m] = 0.0
        w[3 * m:] = np.exp(-rng.random(m) * 30).astype(np.float32)
        w[3 * m + 7] = 1.0
        u_ref = (1.0 + rng.random(4 * m)).astype(np.float32)
        u_ref = np.minimum(u_ref, np.float32(1.9999999))
        u_sys = rng.random(4).astype(np.float32)
        u_vose = rng.random(8 * m).astype(np.float32)
        g["res_w_%d" % m] = w
        g["res_uref_%d" % m], g["res_usys_%d" % m], g["res_uvose_%d" % m] = u_ref, u_sys, u_vose
        g["res_ref_%d" % m] = O.resample(O.RES_REF, w, u_ref, m, 2)
        for ept in ((1,) if m == 32 else (2, 4)):
            if m == 64 and ept == 4:
                continue
            g["res_sys_%d_%d" % (m, ept)] = O.resample(O.RES_SYSTEMATIC, w, u_sys, m, ept)
        g["res_vose_%d" % m] = O.resample(O.RES_VOSE, w, u_vose, m, 2)
        p, a = O.vose_build(w, m)
        g["vose_prob_%d" % m], g["vose_alias_%d" % m] = p, a
    # exchange routing
    for (mode, N, m, t) in ((O.EXCH_RING, 8, 32, 3), (O.EXCH_TORUS, 2048, 512, 2), (O.EXCH_TORUS, 1024, 256, 1),
                            (O.EXCH_TORUS, 12, 64, 4), (O.EXCH_ALL2ALL, 16, 64, 5)):
        keys = np.sort(rng.standard_normal(N * m).astype(np.float32).reshape(N, m), axis=1)[:, ::-1].reshape(-1)
        if mode == O.EXCH_ALL2ALL:
            keys = np.round(keys * 4) / 4  # ties across sub-filters
        tag = "%d_%d_%d_%d" % (mode, N, m, t)
        nx = 4 * t if mode == O.EXCH_TORUS else t
        src = O.exchange_sources(mode, N, m, t, keys).reshape(N, m)
        assert np.array_equal(src[:, :m - nx], np.arange(N * m).reshape(N, m)[:, :m - nx])
        g["exch_src_" + tag] = np.ascontiguousarray(src[:, m - nx:])  # replaced slots only
        if mode == O.EXCH_ALL2ALL:
            g["exch_keys_" + tag] = np.ascontiguousarray(keys, np.float32)
    np.savez_compressed(Path(__file__).with_name("golden.npz"), **g)
    print("wrote", len(g), "arrays")


if __name__ == "__main__":
    main()
