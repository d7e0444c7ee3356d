"""Raw spectral output of a render: the per-pixel invariant intensity
I_nu / nu^3 of every bin (the intensity slots of the reference's ray_matrix,
LttM.jl:176) as a cube [y_pix, x_pix, n_bins], written as NPY (with a JSON
sidecar) or as a FITS primary image. The reference returns only the colour
image after the xyY / RGB conversion (gen_image, LttM.jl:182-208); raw
spectral output ("something like FITS files") is one of its planned
features (the reference's README.md:21).
"""
from __future__ import annotations

import json

import numpy as np


def spectral_cube(spectrum, x_pix: int, y_pix: int, frame: int = 0) -> np.ndarray:
    """[P, N] render output of pixel i + x_pix j (frames concatenated) ->
    [y_pix, x_pix, N] with row 0 at the top of the image (the reference's
    image orientation, rows reversed as in gen_image)."""
    sp = np.asarray(spectrum)
    P = x_pix * y_pix
    cube = sp[frame * P:(frame + 1) * P].reshape(y_pix, x_pix, -1)
    return cube[::-1]


def save_npy(path: str, cube: np.ndarray, colors_nm, meta: dict | None = None) -> None:
    """cube -> path (.npy, float32) and path + '.json' (wavelengths, units, meta)."""
    np.save(path, np.ascontiguousarray(cube, dtype=np.float32))
    side = {"axes": ["y", "x", "bin"], "colors_nm": [float(c) for c in colors_nm],
            "quantity": "invariant intensity I_nu / nu^3 (nu in nm^-1), reference units",
            "meta": meta or {}}
    with open(str(path) + ".json", "w") as f:
        json.dump(side, f, indent=1)


def _card(key: str, value, comment: str = "") -> bytes:
    if isinstance(value, bool):
        v = "T" if value else "F"
        s = f"{key:<8}= {v:>20}"
    elif isinstance(value, (int, np.integer)):
        s = f"{key:<8}= {int(value):>20}"
    elif isinstance(value, (float, np.floating)):
        s = f"{key:<8}= {float(value):>20.12E}"
    else:
        text = str(value).replace("'", "''")
        s = f"{key:<8}= '{text:<8}'"
    if comment:
        s += f" / {comment}"
    return s[:80].ljust(80).encode("ascii")


def save_fits(path: str, cube: np.ndarray, colors_nm, meta: dict | None = None) -> None:
    """cube [y, x, N] -> a FITS primary image (BITPIX -32, NAXIS1 = x, NAXIS2 =
    y, NAXIS3 = bin; big-endian float32). The bin wavelengths go to WAVEnnnn
    cards (nm); meta (short keys) to header cards."""
    cube = np.asarray(cube, dtype=np.float32)
    ny, nx, nb = cube.shape
    cards = [_card("SIMPLE", True, "conforms to FITS"), _card("BITPIX", -32, "IEEE float32"),
             _card("NAXIS", 3), _card("NAXIS1", nx, "x pixels"), _card("NAXIS2", ny, "y pixels"),
             _card("NAXIS3", nb, "spectral bins"), _card("BUNIT", "I_nu/nu^3", "reference units, nu in nm^-1")]
    for i, c in enumerate(colors_nm):
        cards.append(_card(f"WAVE{i:04d}"[:8], float(c), "bin wavelength, nm"))
    for k, v in (meta or {}).items():
        cards.append(_card(str(k).upper()[:8], v))
    cards.append(b"END".ljust(80))
    header = b"".join(cards)
    header += b" " * (-len(header) % 2880)
    # FITS order: NAXIS1 fastest = x, then y (FITS rows run upward), then bin
    data = np.ascontiguousarray(cube[::-1].transpose(2, 0, 1)).astype(">f4").tobytes()
    data += b"\0" * (-len(data) % 2880)
    with open(path, "wb") as f:
        f.write(header)
        f.write(data)


def load_fits(path: str):
    """(cube [y, x, N], header dict) of a file written by save_fits."""
    raw = open(path, "rb").read()
    hdr = {}
    off = 0
    while True:
        card = raw[off:off + 80].decode("ascii")
        off += 80
        key = card[:8].strip()
        if key == "END":
            break
        if card[8:10] == "= ":
            val = card[10:].split(" / ")[0].strip()
            if val.startswith("'"):
                hdr[key] = val.strip("'").rstrip()
            elif val in ("T", "F"):
                hdr[key] = val == "T"
            else:
                hdr[key] = float(val) if any(ch in val for ch in ".E") else int(val)
    off += -off % 2880
    nx, ny, nb = hdr["NAXIS1"], hdr["NAXIS2"], hdr["NAXIS3"]
    data = np.frombuffer(raw[off:off + 4 * nx * ny * nb], dtype=">f4").reshape(nb, ny, nx)
    return data.transpose(1, 2, 0)[::-1].astype(np.float32), hdr


__all__ = ["spectral_cube", "save_npy", "save_fits", "load_fits"]
