"""Generate the golden fixtures under tests/golden/ (run in a container that has
the reference tree; the fixtures are committed, the reference is not needed
afterwards).

vlc_compress_c.json
    The known-answer vectors of the reference's VLC test, the commented-out
    main() at compress.c:546-597 (inputs at :550-553, expected decompressed
    values at :574-577).  They are parsed from the source text here, not typed
    in.  That main() is stale (it calls compress/decompress with 5 arguments,
    compress.h:8-10 declares 6) and was never built, so the fixture also stores
    what the reference's compress.c, compiled by oracle/Makefile, actually
    returns for the same inputs (`reference_outputs`).

soi_small.json
    Outputs of the reference's compute_soi (oracle/_ref/soi_ref_run, built from
    pfft.c + parallel_filter_subsampling.cpp) for small seeded inputs, with a
    sha256 of the exact output bytes and a few sampled values.
"""
import ctypes
import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("SOI_REFERENCE_TREE", "")


def parse_vlc_vectors():
    src = open(os.path.join(REF, "compress.c")).read()
    start = src.index("/*int main()")
    body = src[start:]

    def block(name):
        m = re.search(r"double\s+%s\[2\]\[4\]\s*=\s*\{(.*?)\};" % name, body, re.S)
        rows = re.findall(r"\{([^{}]*)\}", m.group(1))
        return [[float.fromhex(t.strip()) for t in r.split(",") if t.strip()] for r in rows]

    return block("segments"), block("expected")


def aligned(n, dt):
    buf = np.zeros(n + 64, dt)
    off = (-buf.ctypes.data % 64) // buf.itemsize
    return buf[off:off + n]


def vlc_fixture():
    segs, expected = parse_vlc_vectors()
    ref = ctypes.CDLL(os.path.join(REPO, "oracle/_ref/libcompress_ref.so"))
    P = ctypes.c_void_p
    emaxs = []
    for s in segs:
        x = aligned(4, np.float64)
        x[:] = s
        emaxs.append(ref.max_exponent(x.ctypes.data_as(P), 4))
    gmax = max(emaxs)
    outs, words = [], []
    for s, e in zip(segs, emaxs):
        x = aligned(4, np.float64)
        x[:] = s
        o = aligned(64, np.int32)
        n = ref.compress(o.ctypes.data_as(P), x.ctypes.data_as(P), 4, gmax, e, 0)
        d = aligned(4, np.float64)
        ref.decompress(d.ctypes.data_as(P), o.ctypes.data_as(P), 4, gmax, e, None)
        words.append([int(v) for v in o[:n]])
        outs.append([float(v).hex() for v in d])
    return {
        "source": "compress.c:546-597 (inputs :550-553, expected :574-577)",
        "segment_len": 4,
        "inputs": [[float(v).hex() for v in s] for s in segs],
        "expected": [[float(v).hex() for v in s] for s in expected],
        "reference_max_exponent": emaxs,
        "reference_global_max_exponent": gmax,
        "reference_compressed_words": words,
        "reference_outputs": outs,
    }


def soi_fixture():
    cases = []
    run = os.path.join(REPO, "oracle/_ref/soi_ref_run")
    d = tempfile.mkdtemp()
    for (N, P, k, seed, T) in [(2 ** 14, 1, 4, 11, 1), (2 ** 15, 2, 4, 12, 2), (2 ** 16, 1, 16, 13, 4)]:
        rng = np.random.default_rng(seed)
        x = (rng.standard_normal(N) + 1j * rng.standard_normal(N)).astype(np.complex128)
        x.tofile(os.path.join(d, "in.bin"))
        subprocess.run([run, "--N", str(N), "--P", str(P), "--k", str(k), "--threads", str(T),
                        "--in", os.path.join(d, "in.bin"), "--out", os.path.join(d, "out.bin")],
                       check=True, capture_output=True)
        y = np.fromfile(os.path.join(d, "out.bin"), dtype=np.complex128)
        idx = rng.integers(0, N, 16)
        cases.append({
            "N": N, "P": P, "k": k, "S": P * k, "seed": seed,
            "input": "numpy default_rng(seed): standard_normal(N) + 1j*standard_normal(N), complex128",
            "sha256": hashlib.sha256(y.tobytes()).hexdigest(),
            "samples": {str(int(i)): [float(y[i].real).hex(), float(y[i].imag).hex()] for i in idx},
        })
    return {"source": "oracle/_ref/soi_ref_run (pfft.c, parallel_filter_subsampling.cpp)",
            "defaults": "n_mu=5 d_mu=4 B=72 tau=928/1024 sigma=373.7314 (pfft.c:87-91)",
            "cases": cases}


if __name__ == "__main__":
    if not os.path.isfile(os.path.join(REF, "compress.c")):
        sys.exit("set SOI_REFERENCE_TREE to the reference tree (the directory holding compress.c)")
    json.dump(vlc_fixture(), open(os.path.join(HERE, "vlc_compress_c.json"), "w"), indent=1)
    json.dump(soi_fixture(), open(os.path.join(HERE, "soi_small.json"), "w"), indent=1)
    print("wrote fixtures", file=sys.stderr)
