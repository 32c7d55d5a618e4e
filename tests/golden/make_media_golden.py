"""Generates the permeability-file fixture and its golden K.

The file is written in the layout load_permeability reads (main.cpp:918-1032
with LOAD_K_FROM_FILE): a header "Nx Ny" with CRLF, then Ny rows of Nx values
in 14-digit mantissa / 4-digit exponent notation, a blank before positive
values, every value followed by a blank, CRLF line ends.  The values are a
seeded random field written by this script (not taken from the reference).
The golden K is what the reference's own load_permeability, compiled from its
sources into oracle/_ref/capaz_ref_loadk by oracle/Makefile, reads from it.

    python tests/golden/make_media_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LOADK = os.path.join(ROOT, "oracle", "_ref", "capaz_ref_loadk")


def fmt(v: float) -> str:
    """-3.69248837232590E-0001 style (sign column, 4-digit exponent)."""
    m, e = f"{v:.14E}".split("E")
    e = int(e)
    s = f"{m}E{'-' if e < 0 else '+'}{abs(e):04d}"
    return s if v < 0 else " " + s


def write_noise(path: str, values: np.ndarray) -> None:
    ny, nx = values.shape
    with open(path, "wb") as f:
        f.write(f"{nx} {ny}\r\n".encode())
        for j in range(ny):
            f.write(("".join(fmt(v) + " " for v in values[j]) + "\r\n").encode())


def reference_K(noise_path: str, nx: int, ny: int, nz: int) -> np.ndarray:
    with tempfile.TemporaryDirectory() as d:
        run = os.path.join(d, "run")
        os.makedirs(run)
        with open(noise_path, "rb") as src, open(os.path.join(run, "noise.dat"), "wb") as dst:
            dst.write(src.read())
        out = os.path.join(d, "K.bin")
        subprocess.run([LOADK, run, str(nx), str(ny), str(nz), out], check=True, capture_output=True)
        return np.fromfile(out, dtype=np.float64).reshape(nz, ny, nx)


def main():
    if not os.path.exists(LOADK):
        sys.exit("build oracle/_ref/capaz_ref_loadk first (make -C oracle REF=<reference tree> ref)")
    nx, ny = 13, 9
    rng = np.random.default_rng(20)
    vals = rng.normal(0.0, 1.5, size=(ny, nx))
    vals[0, 0] = 0.0
    vals[1, 2] = -1e-3
    vals[2, 3] = 12.5
    noise = os.path.join(HERE, "media_noise_13x9.dat")
    write_noise(noise, vals)
    K = reference_K(noise, nx, ny, 1)
    np.savez_compressed(os.path.join(HERE, "media_K_13x9.npz"), K=K, nx=nx, ny=ny, nz=1)
    print("wrote", noise, "and media_K_13x9.npz", K.min(), K.max())


if __name__ == "__main__":
    main()
