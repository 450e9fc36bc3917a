"""FemState checkpoints in pmsim's JSON layout (byte-compatible with the files pmsim writes).

pmsim serialises ``FemState`` with serde_json (reference ``src/fem/fem_state.rs:217-245``,
fields ``src/fem/fem_state.rs:15-96``): a compact JSON object with the keys in struct order, the
vectors as ``{"data": [...]}``, per cell a ``SecondaryValues`` entry
(``src/fem/secondary_values.rs:8-56``) whose ``solid`` list holds one ``LocalState`` per IP
(``src/material/local_state.rs:9-21``: elastic, int_vars, stress{vec, mandel}, strain or null).
Floats use the shortest round-trip digits in the notation of the ``ryu`` formatter that
serde_json uses (``1.0``, ``0.0123``, ``2.6e-16``, ``1e21``).
"""
from __future__ import annotations

import json

import numpy as np

SCALARS = ["ell", "t", "ddt", "alpha1", "alpha2", "alpha3", "alpha4", "alpha5", "alpha6", "alpha7", "alpha8",
           "beta1", "beta2"]
VECTORS = ["ddu", "u", "v", "a", "u_star", "v_star", "a_star"]


def format_float(x: float) -> str:
    """Shortest round-trip decimal of x in ryu's notation (digits D, value = D x 10^k, kk = len(D) + k):
    k >= 0 and kk <= 16 -> D000.0; 0 < kk <= 16 -> DD.DD; -5 < kk <= 0 -> 0.000D; else D.DDDe(kk-1)."""
    x = float(x)
    if x == 0.0:
        return "-0.0" if np.signbit(x) else "0.0"
    if not np.isfinite(x):
        return "null"  # serde_json writes non-finite floats as null
    r = repr(abs(x))
    sign = "-" if x < 0 else ""
    if "e" in r:
        mant, ex = r.split("e")
        ex = int(ex)
    else:
        mant, ex = r, 0
    if "." in mant:
        ip, fp = mant.split(".")
    else:
        ip, fp = mant, ""
    digits = (ip + fp).lstrip("0")
    k = ex - len(fp)
    # strip trailing zeros of the digit string into the exponent
    stripped = digits.rstrip("0")
    k += len(digits) - len(stripped)
    digits = stripped or "0"
    n = len(digits)
    kk = n + k
    if k >= 0 and kk <= 16:
        out = digits + "0" * k + ".0"
    elif 0 < kk <= 16:
        out = digits[:kk] + "." + digits[kk:]
    elif -5 < kk <= 0:
        out = "0." + "0" * (-kk) + digits
    elif n == 1:
        out = digits + "e" + str(kk - 1)
    else:
        out = digits[0] + "." + digits[1:] + "e" + str(kk - 1)
    return sign + out


def _vec(a) -> str:
    return '{"data":[' + ",".join(format_float(v) for v in np.asarray(a, dtype=float).ravel()) + "]}"


def _tensor(v, mandel) -> str:
    return '{"vec":' + _vec(v) + ',"mandel":"' + mandel + '"}'


def dumps(state: dict) -> str:
    """state: scalars (SCALARS), vectors (VECTORS), and "gauss": list per cell of
    {"ngauss": n, "solid": [{"elastic": bool, "int_vars": [...], "stress": [...], "strain": [...] | None}]},
    "mandel": "Symmetric2D" | "Symmetric"."""
    mandel = state["mandel"]
    parts = [f'"{k}":{format_float(state.get(k, 0.0))}' for k in SCALARS]
    parts += [f'"{k}":{_vec(state.get(k, []))}' for k in VECTORS]
    cells = []
    for c in state["gauss"]:
        ips = []
        for s in c["solid"]:
            strain = "null" if s.get("strain") is None else _tensor(s["strain"], mandel)
            ips.append('{"elastic":' + ("true" if s["elastic"] else "false") + ',"int_vars":' + _vec(s["int_vars"])
                       + ',"stress":' + _tensor(s["stress"], mandel) + ',"strain":' + strain + "}")
        cells.append('{"ngauss":' + str(int(c["ngauss"])) + ',"solid":[' + ",".join(ips) + ']'
                     + ',"porous_liq":[],"porous_liq_gas":[],"porous_sld_liq":[],"porous_sld_liq_gas":[]}')
    parts.append('"gauss":[' + ",".join(cells) + "]")
    return "{" + ",".join(parts) + "}"


def loads(text: str) -> dict:
    d = json.loads(text)
    out = {k: float(d[k]) for k in SCALARS}
    for k in VECTORS:
        out[k] = np.array(d[k]["data"], dtype=float)
    cells = []
    mandel = None
    for c in d["gauss"]:
        ips = []
        for s in c["solid"]:
            mandel = s["stress"]["mandel"]
            ips.append({"elastic": bool(s["elastic"]), "int_vars": list(s["int_vars"]["data"]),
                        "stress": list(s["stress"]["vec"]["data"]),
                        "strain": None if s["strain"] is None else list(s["strain"]["vec"]["data"])})
        cells.append({"ngauss": int(c["ngauss"]), "solid": ips})
    out["gauss"] = cells
    out["mandel"] = mandel or "Symmetric"
    return out


def export_state(elements, u, ddu, t=0.0, ell=1.0, ddt=0.0, strain=None, model_has_int_vars=True) -> str:
    """FemState JSON of an ``Elements`` handle's IP state plus the global vectors u and ddu."""
    sig, ivs, el = elements.get_state()
    ng = elements.ngauss
    mandel = "Symmetric2D" if elements.ndim == 2 else "Symmetric"
    cells = []
    for c in range(elements.mesh.ncell):
        ips = []
        for p in range(ng):
            i = c * ng + p
            ips.append({"elastic": bool(el[i]), "int_vars": list(ivs[i]) if model_has_int_vars else [],
                        "stress": sig[i], "strain": None if strain is None else strain[i]})
        cells.append({"ngauss": ng, "solid": ips})
    st = {k: 0.0 for k in SCALARS}
    st.update(ell=ell, t=t, ddt=ddt, u=u, ddu=ddu, mandel=mandel, gauss=cells)
    return dumps(st)


def import_state(elements, text: str):
    """Loads a FemState JSON into the handle's IP state; returns (u, ddu, t)."""
    st = loads(text)
    ng = elements.ngauss
    nc = elements.ncomp
    sig = np.zeros((elements.nip, nc))
    ivs = np.zeros((elements.nip, 2))
    el = np.ones(elements.nip, np.uint8)
    if len(st["gauss"]) != elements.mesh.ncell:
        raise ValueError("number of cells differs")
    for c, cell in enumerate(st["gauss"]):
        if cell["ngauss"] != ng:
            raise ValueError("number of integration points differs")
        for p, s in enumerate(cell["solid"]):
            i = c * ng + p
            sig[i] = s["stress"]
            iv = s["int_vars"]
            ivs[i, : len(iv)] = iv[:2]
            el[i] = 1 if s["elastic"] else 0
    elements.set_state(sig, ivs, el)
    return st["u"], st["ddu"], st["t"]
