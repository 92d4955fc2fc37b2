"""Fixtures of the headless example program's readers.

Writes a seeded 48x32, 21-label ProbImage file with the reference's own
ProbImage::compress (eps 0.001) and the unaries the reference's decoder +
boostToProb + -log give for it (src/file_storage.cpp:261-285), pinned by
SHA-256; and the seeded image as a 32-bit bottom-up BMP, the layout of the
reference's data/img.bmp.  Needs oracle/_ref (the reference built from its
sources).  Run: python tests/golden/make_cli_golden.py
"""
import ctypes as C
import hashlib
import json
import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from densecrf_ho_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

W, H, L, SEED = 48, 32, 21, 17


def write_bmp32(path, rgb, W, H):
    """32-bit BI_RGB, bottom-up rows, BGRA."""
    px = rgb.reshape(H, W, 3)[::-1, :, ::-1]
    bgra = np.concatenate([px, np.zeros((H, W, 1), np.uint8)], axis=2).astype(np.uint8)
    data = bgra.tobytes()
    hdr = b"BM" + struct.pack("<IHHI", 54 + len(data), 0, 0, 54)
    info = struct.pack("<IiiHHIIiiII", 40, W, H, 1, 32, 0, len(data), 2835, 2835, 0, 0)
    with open(path, "wb") as f:
        f.write(hdr + info + data)


def main():
    lib = O.ref_lib()
    img = synth.make_image(W, H, L, SEED)
    # boosting values (log-probabilities up to a constant) of the image's unaries
    boost = (-img["unary"]).astype(np.float32).reshape(-1)
    cpath = os.path.join(HERE, "cli_48x32.c_unary")
    lib.ref_probimage_compress(W, H, L, boost.ctypes.data_as(C.c_void_p), C.c_float(0.001), cpath.encode())
    w, h, d = C.c_int(), C.c_int(), C.c_int()
    lib.ref_load_unary(cpath.encode(), None, C.byref(w), C.byref(h), C.byref(d))
    out = np.empty(w.value * h.value * d.value, np.float32)
    lib.ref_load_unary(cpath.encode(), out.ctypes.data_as(C.c_void_p), C.byref(w), C.byref(h), C.byref(d))
    write_bmp32(os.path.join(HERE, "cli_48x32.bmp"), img["rgb"], W, H)
    rec = {"W": w.value, "H": h.value, "D": d.value,
           "unary_sha256": hashlib.sha256(out.tobytes()).hexdigest(),
           "rgb_sha256": hashlib.sha256(img["rgb"].tobytes()).hexdigest(),
           "unary_sum": float(out.astype(np.float64).sum())}
    with open(os.path.join(HERE, "cli_48x32.json"), "w") as f:
        json.dump(rec, f, indent=1)
    print(rec)


if __name__ == "__main__":
    main()
