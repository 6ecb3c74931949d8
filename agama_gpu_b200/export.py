"""Write a GPU potential tree as a multi-section Agama-style INI file.

``export_potential(pot, path)`` writes one ``[Potential k]`` section per leaf of
the tree; ``PotentialGPU(path)`` (the factory's INI reader) builds the same tree
back.  Sections:

* analytic leaves: ``type=<Name>`` and the constructor's own parameters;
* Multipole / CylSpline: the coefficient tables inline (``Coefficients`` block, the
  text format ``read_coefs`` parses; values written with 17 significant digits so
  they read back bit for bit).  A Multipole or CylSpline whose node tables were
  replaced on the device (``set_node_tables``) is written with the current ones;
* Evolving: ``type=Evolving``, ``interpLinear``, and a ``Timestamps`` block naming
  one coefficient file per snapshot, written beside the INI file;
* Shifted / Scaled wrappers: ``center=x,y,z`` or ``center=<track file>`` ((T, 4) or
  (T, 7) rows), ``scale=`` / ``ampl=`` or ``scale=<file>`` ((T, 2) or (T, 3) rows) on
  every section below them -- a shift or a scaling of a sum is the sum of the shifted
  or scaled terms.  A Shifted inside a Scaled cannot be written this way (the reader
  applies the scaling first) and raises.

Files beside the INI are named ``<stem>.<k>.*`` after the section that uses them.
"""
from __future__ import annotations

from pathlib import Path
from typing import List, Union

import numpy as np

from .coefs import MultipoleCoefs, coefs_text

_ANALYTIC_TYPES = {
    "NFWPotentialGPU": "NFW", "PlummerPotentialGPU": "Plummer",
    "HernquistPotentialGPU": "Hernquist", "DehnenSphericalPotentialGPU": "Dehnen",
    "IsochronePotentialGPU": "Isochrone", "MiyamotoNagaiPotentialGPU": "MiyamotoNagai",
    "LogHaloPotentialGPU": "LogHalo", "DiskAnsatzPotentialGPU": "DiskAnsatz",
    "UniformAccelerationGPU": "UniformAcceleration",
}


def _fmt(v) -> str:
    return repr(float(v))


def current_multipole_coefs(mp) -> MultipoleCoefs:
    """The coefficient tables of a MultipolePotentialGPU as it evaluates now: the file's
    tables, with the node tables set on the device (set_node_tables) written into their
    columns."""
    c = mp._coefs
    nodes = getattr(mp, "_nodes", None)
    if nodes is None:
        return c
    phi = np.array(c.phi, dtype=np.float64, copy=True)
    dphi = (np.zeros_like(phi) if c.dphi_dr is None
            else np.array(c.dphi_dr, dtype=np.float64, copy=True))
    cols = np.asarray(mp.tables.node_cols)
    phi[:, cols] = nodes[0].detach().to("cpu").numpy()
    dphi[:, cols] = nodes[1].detach().to("cpu").numpy()
    return MultipoleCoefs(np.asarray(c.R_grid, dtype=np.float64).copy(), phi, dphi,
                          list(c.lm_labels), dict(c.params))


def current_cylspline_coefs(cs):
    """The coefficient grids of a CylSplinePotentialGPU as it evaluates now (the grids
    set on the device by set_node_tables, when there were any)."""
    from .coefs import CylSplineCoefs
    grids = cs.__dict__.get("_phi_nodes")
    if grids is None:
        return cs._coefs
    c = cs._coefs
    return CylSplineCoefs(np.asarray(c.R_grid, dtype=np.float64).copy(),
                          np.asarray(c.z_grid, dtype=np.float64).copy(),
                          {m: v.detach().cpu().numpy() for m, v in grids.items()},
                          dict(c.params))


class _Writer:
    def __init__(self, path: Path):
        self.path = path
        self.sections: List[List[str]] = []

    def side_file(self, k: int, tag: str) -> Path:
        return self.path.with_name(f"{self.path.stem}.{k}.{tag}")

    def mod_lines(self, k: int, center, scale) -> List[str]:
        out = []
        if scale is not None:
            arr, ampl = scale
            if arr is None:
                s, a = ampl
                out.append(f"scale={_fmt(s)}")
                if a != 1.0:
                    out.append(f"ampl={_fmt(a)}")
            else:
                f = self.side_file(k, "scale.txt")
                np.savetxt(f, arr, fmt="%.17g")
                out.append(f"scale={f.name}")
                if arr.shape[1] == 2 and ampl[1] != 1.0:
                    out.append(f"ampl={_fmt(ampl[1])}")
        if center is not None:
            c = np.asarray(center, dtype=np.float64)
            if c.ndim == 1:
                out.append("center=" + ",".join(_fmt(v) for v in c))
            else:
                f = self.side_file(k, "center.txt")
                np.savetxt(f, c, fmt="%.17g")
                out.append(f"center={f.name}")
        return out

    def emit(self, pot, center=None, scale=None) -> None:
        from .batch import BatchedPotentialGPU
        from .potentials import (CompositePotentialGPU, CylSplinePotentialGPU,
                                 EvolvingPotentialGPU, MultipolePotentialGPU,
                                 ScaledPotentialGPU, ShiftedPotentialGPU)
        if isinstance(pot, CompositePotentialGPU):
            for c in pot._components:
                self.emit(c, center, scale)
            return
        if isinstance(pot, ShiftedPotentialGPU):
            if scale is not None:
                raise ValueError("a Shifted potential inside a Scaled one cannot be written "
                                 "as INI sections (the reader applies the scaling first)")
            if center is not None:
                raise ValueError("nested Shifted wrappers cannot be written as INI sections")
            self.emit(pot._inner, pot._center_arr, scale)
            return
        if isinstance(pot, ScaledPotentialGPU):
            if scale is not None:
                raise ValueError("nested Scaled wrappers cannot be written as INI sections")
            sc = (pot._scale_arr, (getattr(pot, "_scale_val", 1.0), pot._ampl_val))
            self.emit(pot._inner, center, sc)
            return
        if isinstance(pot, BatchedPotentialGPU):
            raise ValueError("a BatchedPotentialGPU is a set of potentials; export each unit")
        k = len(self.sections) + 1
        head = [f"[Potential {k}]"]
        mods = self.mod_lines(k, center, scale)
        if isinstance(pot, (MultipolePotentialGPU, CylSplinePotentialGPU)):
            coefs = (current_multipole_coefs(pot) if isinstance(pot, MultipolePotentialGPU)
                     else current_cylspline_coefs(pot))
            body = coefs_text(coefs).splitlines()[1:]          # drop its own [Potential]
            at = next(i for i, ln in enumerate(body) if ln.strip().lower() == "coefficients")
            self.sections.append(head + body[:at] + mods + body[at:])
            return
        if isinstance(pot, EvolvingPotentialGPU):
            lines = head + ["type=Evolving", f"interpLinear={1 if pot._interpolate else 0}"] + mods
            lines.append("Timestamps")
            for i, (t, p) in enumerate(zip(pot._times, pot._pots)):
                if not isinstance(p, (MultipolePotentialGPU, CylSplinePotentialGPU)):
                    raise ValueError("Evolving snapshots must be Multipole or CylSpline to export")
                coefs = (current_multipole_coefs(p) if isinstance(p, MultipolePotentialGPU)
                         else current_cylspline_coefs(p))
                f = self.side_file(k, f"snap{i}.coef")
                f.write_text(coefs_text(coefs))
                lines.append(f"{_fmt(t)}\t{f.name}")
            self.sections.append(lines)
            return
        name = _ANALYTIC_TYPES.get(type(pot).__name__)
        if name is None or not hasattr(pot, "_init_args"):
            raise ValueError(f"cannot export {type(pot).__name__}")
        lines = head + [f"type={name}"]
        for key, v in pot._init_args.items():
            lines.append(f"{key}={_fmt(v)}")
        self.sections.append(lines + mods)


def export_potential(pot, path: Union[str, Path]) -> Path:
    """Write ``pot`` as a multi-section INI file (plus side files next to it); returns the
    INI path.  ``PotentialGPU(path)`` reads it back."""
    path = Path(path)
    w = _Writer(path)
    w.emit(pot)
    if not w.sections:
        raise ValueError("nothing to export")
    path.write_text("\n\n".join("\n".join(s) for s in w.sections) + "\n")
    return path
