"""The reference's binary restart / snapshot format (read_state.cpp:3-94,
write_state.cpp:3-63, output.cpp:3-16).

Layout: a 124-byte header written field by field (no padding):

    int n_bodies, int nnopt, double hmin, hmax, sep0, t_end, dt_out,
    int snapshot_number, int iteration_number, double global_time, int nav,
    double alpha, beta, eta2, int ngr, int nrelax, double trelax, dt, omega2

then 23 doubles per particle:

    x y z m h rho vx vy vz ax ay az u du gx gy gz phi mu_grams aa bb cc divv

with h = range / 2 (read_state.cpp:42 doubles it, write_state.cpp:34 halves
it) and mu stored in grams (mu * 1.66054e-24, read_state.cpp:61).  aa, bb, cc
are written as -1 (write_state.cpp:57-60).  The particle dicts use this
package's field names (range = 2h, mu dimensionless).
"""
from __future__ import annotations

import numpy as np

AMU = 1.66054e-24
HEADER = np.dtype([
    ("n_bodies", "<i4"), ("nnopt", "<i4"), ("hmin", "<f8"), ("hmax", "<f8"), ("sep0", "<f8"), ("t_end", "<f8"),
    ("dt_out", "<f8"), ("snapshot_number", "<i4"), ("iteration_number", "<i4"), ("global_time", "<f8"),
    ("nav", "<i4"), ("alpha", "<f8"), ("beta", "<f8"), ("eta2", "<f8"), ("ngr", "<i4"), ("nrelax", "<i4"),
    ("trelax", "<f8"), ("dt", "<f8"), ("omega2", "<f8"),
])
assert HEADER.itemsize == 124
PARTICLE = ("x", "y", "z", "m", "h", "rho", "vx", "vy", "vz", "ax", "ay", "az", "u", "du", "gx", "gy", "gz", "phi",
            "mu_g", "aa", "bb", "cc", "divv")


def default_header(n: int, **kw) -> dict:
    h = {k: 0 for k in HEADER.names}
    h.update(n_bodies=n, t_end=1e30, dt_out=0.0, alpha=1.0, beta=2.0)
    h.update(kw)
    return h


def read_state(path: str):
    """Return (header dict, particle dict) from a restart/snapshot file."""
    with open(path, "rb") as f:
        raw = f.read()
    if len(raw) < HEADER.itemsize:
        raise ValueError(f"{path}: truncated header ({len(raw)} bytes)")
    hdr = np.frombuffer(raw[:HEADER.itemsize], HEADER)[0]
    header = {k: hdr[k].item() for k in HEADER.names}
    n = header["n_bodies"]
    if n < 0:
        raise ValueError(f"{path}: negative particle count {n}")
    need = HEADER.itemsize + 23 * 8 * n
    if len(raw) < need:
        raise ValueError(f"{path}: truncated body ({len(raw)} of {need} bytes)")
    body = np.frombuffer(raw[HEADER.itemsize:need], "<f8").reshape(n, 23)
    p = {k: body[:, c].copy() for c, k in enumerate(PARTICLE)}
    p["range"] = 2.0 * p.pop("h")
    p["mu"] = p.pop("mu_g") / AMU
    for k in ("aa", "bb", "cc"):
        p.pop(k)
    p["dt"] = header["dt"]
    p["time"] = header["global_time"]
    return header, p


def write_state(path: str, header: dict, p: dict):
    """Write a restart/snapshot file (write_state.cpp:3-63)."""
    n = int(np.asarray(p["x"]).size)
    h = dict(header)
    h["n_bodies"] = n
    hdr = np.zeros(1, HEADER)
    for k in HEADER.names:
        hdr[k] = h.get(k, 0)
    body = np.empty((n, 23), "<f8")
    cols = dict(p)
    cols["h"] = 0.5 * np.asarray(p["range"], np.float64)
    cols["mu_g"] = np.asarray(p["mu"], np.float64) * AMU
    for c, k in enumerate(PARTICLE):
        if k in ("aa", "bb", "cc"):
            body[:, c] = -1.0
        else:
            body[:, c] = np.asarray(cols.get(k, np.zeros(n)), np.float64)
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        f.write(body.tobytes())
