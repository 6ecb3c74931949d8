"""Agama coefficient-file reader and writer (Multipole and CylSpline text format).

The reference does not ship its reader: it imports ``read_coefs`` from the
external ``nbody_streams.agama_helper`` package (gpu_potential.py:680-686,
1307-1313, 2219-2222), which is not vendored.  This module is written from the
file format itself, as Agama exports it and as the reference's fixtures show
(tests/600.dark.none_8.coef_mul_DR, tests/100.LMC.none_8.coef_mult,
tests/600.bar.none_8.coef_cylsp_DR):

Multipole::

    [Potential]
    type=Multipole
    gridSizeR=25
    lmax=8
    Coefficients
    #Phi
    #radius  l=0,m=0  l=1,m=-1 ...        <- one column per (l,m), m = -l..l
    r_0      Phi_00   Phi_1-1 ...
    ...
    #dPhi/dr
    #radius  l=0,m=0 ...
    r_0      dPhi_00/dr ...

CylSpline::

    [Potential]
    type=CylSpline
    gridSizeR=25
    gridSizez=49
    mmax=8
    Coefficients
    #Phi
    -8  #m
    #R(row)\\z(col)  z_0  z_1 ...
    R_0  Phi_m(R_0, z_0) ...
    ...
    -7  #m
    ...

``read_coefs`` accepts a path or the text of one ``[Potential]`` section (the
reference passes inline INI sections as text, gpu_potential.py:2219-2224).
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field
from pathlib import Path
from typing import Dict, Iterable, List, Optional, Tuple, Union

import numpy as np

__all__ = ["MultipoleCoefs", "CylSplineCoefs", "read_coefs", "write_coefs"]


@dataclass
class MultipoleCoefs:
    """Radial tables of a Multipole expansion.

    R_grid   : (nR,) radii
    phi      : (nR, n_lm) Phi_lm(r), columns in ``lm_labels`` order
    dphi_dr  : (nR, n_lm) dPhi_lm/dr, or None when the file has no derivative block
    lm_labels: list of (l, m)
    """
    R_grid: np.ndarray
    phi: np.ndarray
    dphi_dr: Optional[np.ndarray]
    lm_labels: List[Tuple[int, int]]
    params: Dict[str, str] = field(default_factory=dict)

    @property
    def lmax(self) -> int:
        return max(l for l, _ in self.lm_labels)

    def zeroed(self, keep_lm: Iterable[Tuple[int, int]]) -> "MultipoleCoefs":
        """Copy with every column not in ``keep_lm`` set to zero."""
        keep = {(int(l), int(m)) for l, m in keep_lm}
        mask = np.array([(l, m) in keep for l, m in self.lm_labels])
        phi = self.phi * mask[None, :]
        d = None if self.dphi_dr is None else self.dphi_dr * mask[None, :]
        return MultipoleCoefs(self.R_grid.copy(), phi, d, list(self.lm_labels), dict(self.params))


@dataclass
class CylSplineCoefs:
    """Meridional-plane tables of a CylSpline expansion.

    R_grid : (nR,) cylindrical radii
    z_grid : (nz,) heights (full range, or z >= 0 only)
    phi    : {m: (nR, nz)} Fourier amplitude of harmonic m (m < 0: sin terms)
    """
    R_grid: np.ndarray
    z_grid: np.ndarray
    phi: Dict[int, np.ndarray]
    params: Dict[str, str] = field(default_factory=dict)

    @property
    def mmax(self) -> int:
        return max(abs(m) for m in self.phi)


_LM_RE = re.compile(r"l\s*=\s*(-?\d+)\s*,\s*m\s*=\s*(-?\d+)")


def _split_header(lines: List[str]) -> Tuple[Dict[str, str], int]:
    """key=value lines up to 'Coefficients'; returns (params, index after it)."""
    params: Dict[str, str] = {}
    for i, ln in enumerate(lines):
        s = ln.strip()
        if not s or s.startswith("[") or s.startswith(";"):
            continue
        if s.lower() == "coefficients":
            return params, i + 1
        if s.startswith("#"):
            continue
        if "=" in s:
            k, _, v = s.partition("=")
            params[k.strip().lower()] = v.split("#")[0].strip()
    raise ValueError("coefficient text has no 'Coefficients' block")


def _floats(s: str) -> List[float]:
    return [float(t) for t in s.split()]


def _read_multipole(lines: List[str], params: Dict[str, str]) -> MultipoleCoefs:
    blocks: Dict[str, Tuple[List[Tuple[int, int]], List[List[float]]]] = {}
    cur = None
    labels: List[Tuple[int, int]] = []
    for ln in lines:
        s = ln.strip()
        if not s:
            continue
        if s.startswith("["):
            break
        if s.startswith("#"):
            body = s[1:].strip()
            lm = _LM_RE.findall(body)
            if lm:
                labels = [(int(l), int(m)) for l, m in lm]
                if cur is not None:
                    blocks[cur] = (labels, [])
            else:
                key = body.split()[0].lower() if body else ""
                cur = "phi" if key == "phi" else ("dphi" if key.startswith("dphi") else key)
            continue
        if cur is None or cur not in blocks:
            raise ValueError(f"numeric row outside a labelled block: {s[:60]!r}")
        blocks[cur][1].append(_floats(s))
    if "phi" not in blocks:
        raise ValueError("Multipole coefficients have no #Phi block")
    lab, rows = blocks["phi"]
    arr = np.asarray(rows, dtype=np.float64)
    if arr.ndim != 2 or arr.shape[1] != len(lab) + 1:
        raise ValueError(f"#Phi block has shape {arr.shape}, expected (nR, {len(lab) + 1})")
    R = arr[:, 0].copy()
    phi = np.ascontiguousarray(arr[:, 1:])
    dphi = None
    if "dphi" in blocks:
        lab2, rows2 = blocks["dphi"]
        arr2 = np.asarray(rows2, dtype=np.float64)
        if arr2.shape != arr.shape or lab2 != lab:
            raise ValueError("#dPhi/dr block does not match the #Phi block")
        if not np.allclose(arr2[:, 0], R, rtol=1e-12, atol=0):
            raise ValueError("#dPhi/dr radii differ from #Phi radii")
        dphi = np.ascontiguousarray(arr2[:, 1:])
    return MultipoleCoefs(R, phi, dphi, list(lab), params)


def _read_cylspline(lines: List[str], params: Dict[str, str]) -> CylSplineCoefs:
    phi: Dict[int, np.ndarray] = {}
    z_grid: Optional[np.ndarray] = None
    R_rows: Optional[np.ndarray] = None
    m_cur: Optional[int] = None
    rows: List[List[float]] = []
    in_phi = False

    def flush():
        nonlocal R_rows
        if m_cur is None:
            return
        arr = np.asarray(rows, dtype=np.float64)
        if arr.ndim != 2 or z_grid is None or arr.shape[1] != len(z_grid) + 1:
            raise ValueError(f"CylSpline block m={m_cur} has shape {arr.shape}")
        if R_rows is None:
            R_rows = arr[:, 0].copy()
        elif arr.shape[0] != len(R_rows) or not np.allclose(arr[:, 0], R_rows, rtol=1e-12):
            raise ValueError(f"CylSpline block m={m_cur}: R grid differs from earlier blocks")
        phi[m_cur] = np.ascontiguousarray(arr[:, 1:])

    for ln in lines:
        s = ln.strip()
        if not s:
            continue
        if s.startswith("["):
            break
        if s.startswith("#"):
            body = s[1:].strip()
            low = body.lower()
            if low.startswith("phi"):
                in_phi = True
                continue
            if low.startswith("r(row)") or low.startswith("r (row)"):
                zs = _floats(body.split(None, 1)[1]) if len(body.split(None, 1)) > 1 else []
                zarr = np.asarray(zs, dtype=np.float64)
                if z_grid is None:
                    z_grid = zarr
                elif zarr.shape != z_grid.shape or not np.allclose(zarr, z_grid, rtol=1e-12):
                    raise ValueError("CylSpline z grid differs between blocks")
                continue
            # any other '#...' title (e.g. '#dPhi/dR') ends the Phi data
            if in_phi and m_cur is not None:
                flush()
                m_cur = None
                rows = []
            in_phi = False
            continue
        if not in_phi:
            continue
        if "#m" in s:
            flush()
            m_cur = int(float(s.split("#")[0].strip()))
            rows = []
            continue
        rows.append(_floats(s))
    if in_phi:
        flush()
    if not phi or z_grid is None or R_rows is None:
        raise ValueError("CylSpline coefficients have no #Phi data")
    return CylSplineCoefs(R_rows, z_grid, phi, params)


def _text_of(src: Union[str, Path]) -> str:
    if isinstance(src, Path):
        return src.read_text()
    s = str(src)
    if "\n" in s and ("coefficients" in s.lower() or s.lstrip().startswith("[")):
        return s
    return Path(s).read_text()


def read_coefs(src: Union[str, Path]) -> Union[MultipoleCoefs, CylSplineCoefs]:
    """Parse an Agama Multipole or CylSpline coefficient file (path or text)."""
    text = _text_of(src)
    lines = text.splitlines()
    params, start = _split_header(lines)
    typ = params.get("type", "").lower().replace("_", "").replace(" ", "")
    if typ == "multipole":
        return _read_multipole(lines[start:], params)
    if typ == "cylspline":
        return _read_cylspline(lines[start:], params)
    raise ValueError(f"unsupported coefficient type {params.get('type')!r}")


def _fmt(v: float) -> str:
    return repr(float(v))


def write_coefs(path: Union[str, Path], coefs: Union[MultipoleCoefs, CylSplineCoefs]) -> None:
    """Write coefficients in the same text format (round-trips through read_coefs)."""
    Path(path).write_text(coefs_text(coefs))


def coefs_text(coefs: Union[MultipoleCoefs, CylSplineCoefs]) -> str:
    """The coefficient file's text: a [Potential] section with inline Coefficients."""
    out: List[str] = ["[Potential]"]
    if isinstance(coefs, MultipoleCoefs):
        lmax = coefs.lmax
        out += ["type=Multipole", f"gridSizeR={len(coefs.R_grid)}", f"lmax={lmax}",
                "symmetry=None", "Coefficients", "#Phi"]
        hdr = "#radius\t" + "\t".join(f"l={l},m={m}" for l, m in coefs.lm_labels)
        out.append(hdr)
        for i, r in enumerate(coefs.R_grid):
            out.append("\t".join([_fmt(r)] + [_fmt(v) for v in coefs.phi[i]]))
        if coefs.dphi_dr is not None:
            out += ["", "#dPhi/dr", hdr]
            for i, r in enumerate(coefs.R_grid):
                out.append("\t".join([_fmt(r)] + [_fmt(v) for v in coefs.dphi_dr[i]]))
    else:
        out += ["type=CylSpline", f"gridSizeR={len(coefs.R_grid)}",
                f"gridSizez={len(coefs.z_grid)}", f"mmax={coefs.mmax}", "symmetry=None",
                "Coefficients", "#Phi"]
        for m in sorted(coefs.phi):
            out.append(f"{m}\t#m")
            out.append("#R(row)\\z(col)\t" + "\t".join(_fmt(z) for z in coefs.z_grid))
            tab = coefs.phi[m]
            for i, R in enumerate(coefs.R_grid):
                out.append("\t".join([_fmt(R)] + [_fmt(v) for v in tab[i]]))
    return "\n".join(out) + "\n"
