"""The input file of ed_read_input (src/INPUT_VARS.f90:87-193), read on the host.

One `KEY=value` per line as SciFortran's parse_input_variable reads it: keys are case
insensitive, `!` starts a comment, Fortran reals (`1.d-9`, `2D0`), logicals (`T`, `.false.`)
and comma-separated lists are accepted; keys that are absent keep the reference's defaults.
Only the keys that shape the hot path are turned into objects here (`model_from_input`,
`diag_params`); the rest are returned as read.
"""
from __future__ import annotations

import re

from . import _edgpu_lib as L
from .diag import DiagParams
from .edlat import Model

# key -> default, as declared in src/INPUT_VARS.f90:106-166 (lists per orbital, Norb=1)
DEFAULTS = {
    "NORB": 1, "NSITES": [1], "NSPIN": 1, "ED_FILLING": 0, "ULOC": [2.0], "UST": 0.0, "JH": 0.0, "JX": 0.0,
    "JP": 0.0, "TEMP": 0.001, "ED_FINITE_TEMP": False, "XMU": 0.0, "SB_FIELD": 0.1, "WINI": -5.0, "WFIN": 5.0,
    "LMATS": 4096, "LREAL": 5000, "LTAU": 1024, "GF_FLAG": [False], "CHISPIN_FLAG": [False], "OC_FLAG": [False],
    "DM_FLAG": False, "RDM_FLAG": False, "OFFDIAG_GF_FLAG": False, "OFFDIAG_CHISPIN_FLAG": False, "HFMODE": True,
    "EPS": 0.01, "CUTOFF": 1e-9, "GS_THRESHOLD": 1e-9, "ED_METHOD": "lanczos", "ED_TWIN": False,
    "ED_SPARSE_H": True, "ED_PRINT_G": True, "ED_PRINT_DM": False, "ED_VERBOSE": 3, "LANC_METHOD": "arpack",
    "LANC_NSTATES_SECTOR": 2, "LANC_NCV_FACTOR": 10, "LANC_NCV_ADD": 0, "LANC_NITER": 512, "LANC_NGFITER": 200,
    "LANC_TOLERANCE": 1e-18, "LANC_DIM_THRESHOLD": 1024, "LOGFILE": 6,
}


def _scalar(tok: str, like):
    tok = tok.strip().strip("'\"")
    if isinstance(like, bool):
        t = tok.lower().strip(".")
        if t in ("t", "true"):
            return True
        if t in ("f", "false"):
            return False
        raise ValueError(f"not a logical: {tok!r}")
    if isinstance(like, int):
        return int(tok)
    if isinstance(like, float):
        return float(re.sub(r"[dD]", "e", tok))
    return tok


def _value(text: str, default):
    if isinstance(default, list):
        return [_scalar(t, default[0]) for t in text.split(",") if t.strip()]
    return _scalar(text, default)


def read_input(path: str) -> dict:
    """All keys of DEFAULTS, overridden by the file; unknown keys are kept as strings."""
    cfg = {k: (list(v) if isinstance(v, list) else v) for k, v in DEFAULTS.items()}
    with open(path) as f:
        for lineno, raw in enumerate(f, 1):
            line = raw.split("!", 1)[0].strip()
            if not line or "=" not in line:
                continue
            key, text = line.split("=", 1)
            key = key.strip().upper()
            if key in DEFAULTS:
                try:
                    cfg[key] = _value(text, DEFAULTS[key])
                except ValueError as exc:
                    raise L.EdgError(L.EDG_ERR_ARG, "ed_read_input", f"{path}:{lineno}: {key}: {exc}") from None
            else:
                cfg[key] = text.strip()
    if cfg["NORB"] != 1:
        raise L.EdgError(L.EDG_ERR_UNSUPPORTED, "ed_read_input", "NORB > 1 is outside the device engine")
    return cfg


def model_from_input(cfg: dict, hij) -> Model:
    """Model of the hot path from the keys ULOC, XMU, HFMODE, ED_FILLING and a hopping matrix
    (from Hij_read or a lattice builder)."""
    return Model(hij, uloc=float(cfg["ULOC"][0]), xmu=float(cfg["XMU"]), hfmode=bool(cfg["HFMODE"]),
                 ed_filling=int(cfg["ED_FILLING"]))


def sector_form(cfg: dict) -> int:
    """ED_SPARSE_H: stored (T) or direct (F) H x v."""
    return L.EDG_FORM_STORED if cfg["ED_SPARSE_H"] else L.EDG_FORM_DIRECT


def diag_params(cfg: dict, lanc_tolerance: float | None = None) -> DiagParams:
    """DiagParams from the keys of the diagonalisation step. LANC_TOLERANCE is ARPACK's
    relative tolerance in the reference (1e-18 asks for machine precision); here it bounds
    the Lanczos residual, so values below 1e-12 are raised to 1e-12 unless given."""
    tol = lanc_tolerance if lanc_tolerance is not None else max(float(cfg["LANC_TOLERANCE"]), 1e-12)
    return DiagParams(finite_temp=bool(cfg["ED_FINITE_TEMP"]), temp=float(cfg["TEMP"]), cutoff=float(cfg["CUTOFF"]),
                      gs_threshold=float(cfg["GS_THRESHOLD"]), lanc_method=str(cfg["LANC_METHOD"]).lower(),
                      lanc_nstates_sector=int(cfg["LANC_NSTATES_SECTOR"]), lanc_niter=int(cfg["LANC_NITER"]),
                      lanc_tolerance=tol, lanc_dim_threshold=int(cfg["LANC_DIM_THRESHOLD"]),
                      ed_twin=bool(cfg["ED_TWIN"]))
