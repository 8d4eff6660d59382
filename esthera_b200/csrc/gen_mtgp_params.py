#!/usr/bin/env python3
"""Regenerate ``mtgp32_params_11213.inc`` from the MTGP32-11213 parameter table.

The 200 MTGP32-11213 parameter sets are data produced by the MTGP dynamic
creator (Saito & Matsumoto, Hiroshima University, BSD-3).  Reproducing the
reference's random streams bit for bit requires the *same* parameter sets, so
this script reads them from the reference tree
(``src/partfilt/cuda/mtgp/mtgp32dc-param-11213.c``) and writes them in this
project's own flat layout: for each set, 52 uint32 words

    [0] pos  [1] sh1  [2] sh2  [3] mask
    [4..19]  tbl[16]          (recursion matrix)
    [20..35] tmp_tbl[16]      (uint32 tempering)
    [36..51] flt_tmp_tbl[16]  (tempering + conversion to float in [1,2))

Usage: python gen_mtgp_params.py <path-to-mtgp32dc-param-11213.c> [out.inc]
"""
import re
import sys
from pathlib import Path

WORDS_PER_SET = 52

LICENSE = """\
/*
 * MTGP32-11213 parameter sets (200 sets), regenerated by gen_mtgp_params.py.
 *
 * Copyright (c) 2009, 2010 Mutsuo Saito, Makoto Matsumoto and Hiroshima
 * University.  All rights reserved.
 *
 * Redistribution and use in source and binary forms, with or without
 * modification, are permitted provided that the following conditions are
 * met:
 *
 *     * Redistributions of source code must retain the above copyright
 *       notice, this list of conditions and the following disclaimer.
 *     * Redistributions in binary form must reproduce the above
 *       copyright notice, this list of conditions and the following
 *       disclaimer in the documentation and/or other materials provided
 *       with the distribution.
 *     * Neither the name of the Hiroshima University nor the names of
 *       its contributors may be used to endorse or promote products
 *       derived from this software without specific prior written
 *       permission.
 *
 * THIS SOFTWARE IS PROVIDED BY THE COPYRIGHT HOLDERS AND CONTRIBUTORS
 * "AS IS" AND ANY EXPRESS OR IMPLIED WARRANTIES, INCLUDING, BUT NOT
 * LIMITED TO, THE IMPLIED WARRANTIES OF MERCHANTABILITY AND FITNESS FOR
 * A PARTICULAR PURPOSE ARE DISCLAIMED. IN NO EVENT SHALL THE COPYRIGHT
 * OWNER OR CONTRIBUTORS BE LIABLE FOR ANY DIRECT, INDIRECT, INCIDENTAL,
 * SPECIAL, EXEMPLARY, OR CONSEQUENTIAL DAMAGES (INCLUDING, BUT NOT
 * LIMITED TO, PROCUREMENT OF SUBSTITUTE GOODS OR SERVICES; LOSS OF USE,
 * DATA, OR PROFITS; OR BUSINESS INTERRUPTION) HOWEVER CAUSED AND ON ANY
 * THEORY OF LIABILITY, WHETHER IN CONTRACT, STRICT LIABILITY, OR TORT
 * (INCLUDING NEGLIGENCE OR OTHERWISE) ARISING IN ANY WAY OUT OF THE USE
 * OF THIS SOFTWARE, EVEN IF ADVISED OF THE POSSIBILITY OF SUCH DAMAGE.
 *
 * Layout per set (52 words): pos, sh1, sh2, mask, tbl[16], tmp_tbl[16],
 * flt_tmp_tbl[16].  Included as the initialiser of a uint32_t array.
 */
"""


def parse(path):
    src = Path(path).read_text()
    blocks = src.split("/* No.")[1:]
    sets = []
    for b in blocks:
        body = b.split("*/", 1)[1]
        ints = [int(v) for v in re.findall(r"^\s*(\d+),\s*$", body, re.M)[:4]]
        mexp, pos, sh1, sh2 = ints
        if mexp != 11213:
            raise ValueError("unexpected mexp %d" % mexp)
        words = [int(v, 16) for v in re.findall(r"UINT32_C\((0x[0-9a-fA-F]+)\)", body)]
        if len(words) < 49:
            raise ValueError("short parameter block")
        tbl, tmp, flt, mask = words[0:16], words[16:32], words[32:48], words[48]
        sets.append([pos, sh1, sh2, mask] + tbl + tmp + flt)
    if len(sets) != 200:
        raise ValueError("expected 200 parameter sets, found %d" % len(sets))
    return sets


def main():
    src = sys.argv[1]
    out = Path(sys.argv[2]) if len(sys.argv) > 2 else Path(__file__).with_name("mtgp32_params_11213.inc")
    sets = parse(src)
    lines = [LICENSE]
    for i, s in enumerate(sets):
        assert len(s) == WORDS_PER_SET
        lines.append("/* set %d */" % i)
        for k in range(0, WORDS_PER_SET, 4):
            lines.append("  " + ", ".join("0x%08xu" % w for w in s[k:k + 4]) + ",")
    out.write_text("\n".join(lines) + "\n")
    print("wrote", out, len(sets), "sets")


if __name__ == "__main__":
    main()
