"""Checkpoint / restart in the reference's on-disk layout.

The reference saves the solution every ``checkpoint_dt`` of simulated time
(``Simulation.cpp:1084-1116``) and restarts from a given cycle
(``Simulation.cpp:350-388``):

* ``<folder>/Cycle<ti>/checkpoint_cycle_<ti>.<rank:08d>.chk``: the rank's part
  of the solution as ``ParGridFunction::Save`` writes it, i.e. MFEM's text
  grid-function format: a ``FiniteElementSpace`` header naming the element
  collection (``L2_T1_<d>D_P<N>``: discontinuous, Gauss-Lobatto basis,
  ``Simulation.hpp:63``), ``VDim`` (the nv conserved variables), ``Ordering``
  (0 = byNODES, ``Simulation.hpp:64``), a blank line, then one value per line;
* ``<folder>/Cycle<ti>/checkpoint_cycle_<ti>.json``: ``{"time": t, "cycle":
  ti}``, written by rank 0; on load the cycle in it must equal the requested
  one (``Simulation.cpp:367``).

The values are the byNODES state this library computes on (node = element *
Np^d + lexicographic node index, elements in the mesh's order), so a
single-rank reference checkpoint of a Cartesian mesh loads straight into
``DGSEMOperator`` and a checkpoint written here restarts the reference.  The
reference writes with the stream's default six significant digits, so its
checkpoints are rounded; :func:`save` writes 17 significant digits (exact
round trip) unless ``precision`` says otherwise.  With several ranks each
rank saves and loads its own elements (``SlabDecomposition`` owned elements
here; the reference's METIS partition there), so multi-rank files only
restart the decomposition that wrote them.
"""
from __future__ import annotations

import json
import os
import re
from dataclasses import dataclass

import numpy as np

_FEC = re.compile(r"^(?:L2|DG)_(?:T(\d+)_)?(\d)D_P(\d+)$")
GAUSS_LOBATTO = 1  # MFEM BasisType::GaussLobatto


@dataclass
class Checkpoint:
    u: np.ndarray   # byNODES state, float64
    time: float
    cycle: int
    dim: int
    order: int


def paths(folder: str, cycle: int, rank: int = 0):
    """(solution file, meta file) of a cycle, named as Simulation.cpp:1088-1104."""
    d = os.path.join(folder, f"Cycle{int(cycle)}")
    return (os.path.join(d, f"checkpoint_cycle_{int(cycle)}.{int(rank):08d}.chk"),
            os.path.join(d, f"checkpoint_cycle_{int(cycle)}.json"))


def _host(u) -> np.ndarray:
    if hasattr(u, "detach"):  # torch tensor (device or host)
        u = u.detach().cpu().numpy()
    a = np.ascontiguousarray(u, dtype=np.float64).reshape(-1)
    return a


def write_gridfunction(f, u, dim: int, order: int, precision: int = 17) -> None:
    """MFEM's grid-function text format for a DG Gauss-Lobatto space of
    dim + 2 variables in byNODES order (GridFunction::Save)."""
    a = _host(u)
    nv = dim + 2
    if a.size % (nv * (order + 1) ** dim):
        raise ValueError(f"{a.size} values are not whole elements of {nv} variables at order {order}")
    f.write("FiniteElementSpace\n")
    f.write(f"FiniteElementCollection: L2_T{GAUSS_LOBATTO}_{dim}D_P{order}\n")
    f.write(f"VDim: {nv}\n")
    f.write("Ordering: 0\n\n")
    fmt = f"%.{int(precision)}g"
    np.savetxt(f, a, fmt=fmt)


def read_gridfunction(f):
    """Parses MFEM's grid-function text format; returns (dim, order, u) with
    u in byNODES order (a byVDIM file is reordered)."""
    head = {}
    line = f.readline()
    if line.strip() != "FiniteElementSpace":
        raise ValueError(f"not an MFEM grid function (first line {line.strip()!r})")
    while True:
        line = f.readline()
        if not line:
            raise ValueError("grid function ends inside its header")
        if not line.strip():
            break
        key, _, val = line.partition(":")
        head[key.strip()] = val.strip()
    m = _FEC.match(head.get("FiniteElementCollection", ""))
    if not m:
        raise ValueError(f"unsupported element collection {head.get('FiniteElementCollection')!r}")
    btype = int(m.group(1)) if m.group(1) is not None else 0
    if btype != GAUSS_LOBATTO:
        raise ValueError(f"basis type {btype}: this library's nodes are Gauss-Lobatto (type {GAUSS_LOBATTO})")
    dim, order = int(m.group(2)), int(m.group(3))
    vdim = int(head.get("VDim", "1"))
    if vdim != dim + 2:
        raise ValueError(f"VDim {vdim}: expected {dim + 2} conserved variables in {dim}D")
    ordering = int(head.get("Ordering", "0"))
    vals = np.array(f.read().split(), dtype=np.float64)
    nper = vdim * (order + 1) ** dim
    if vals.size == 0 or vals.size % nper:
        raise ValueError(f"{vals.size} values are not whole elements of {nper}")
    if ordering == 1:  # byVDIM: variables interleaved per node
        vals = np.ascontiguousarray(vals.reshape(-1, vdim).T).reshape(-1)
    elif ordering != 0:
        raise ValueError(f"unknown ordering {ordering}")
    return dim, order, vals


def save(folder: str, cycle: int, time: float, u, dim: int, order: int, rank: int = 0,
         precision: int = 17, write_meta: bool | None = None) -> str:
    """Writes cycle ``cycle`` (the solution file of ``rank``; the meta file
    from rank 0 unless ``write_meta`` says otherwise).  Returns the solution
    file's path."""
    chk, meta = paths(folder, cycle, rank)
    os.makedirs(os.path.dirname(chk), exist_ok=True)
    with open(chk, "w") as f:
        write_gridfunction(f, u, dim, order, precision)
    if write_meta if write_meta is not None else rank == 0:
        with open(meta, "w") as f:
            f.write("{\n \"time\": %s,\n \"cycle\": %d\n}\n" % (repr(float(time)), int(cycle)))
    return chk


def load(folder: str, cycle: int, rank: int = 0) -> Checkpoint:
    """Reads cycle ``cycle`` for ``rank``; the meta file's cycle must match."""
    if int(cycle) <= 0:
        raise ValueError("invalid cycle number (the reference requires cycle > 0)")
    chk, meta = paths(folder, cycle, rank)
    with open(meta) as f:
        J = json.load(f)
    t, ti = float(J.get("time", 0.0)), int(J.get("cycle", 0))
    if ti != int(cycle):
        raise ValueError(f"meta file {meta} holds cycle {ti}, not {cycle}")
    with open(chk) as f:
        dim, order, u = read_gridfunction(f)
    return Checkpoint(u, t, ti, dim, order)
