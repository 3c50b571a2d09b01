"""What a run writes as it goes: DCD frames, the StateDataReporter log, and
`.rst` checkpoints, in the formats the reference writes and reads
(src/analysis/dcd.ts, src/analysis/log.ts, src/engine/state.ts:203).

DCD is CHARMM's Fortran-unformatted dialect as OpenMM writes it
(`openmm/app/dcdfile.py`): every record between 4-byte length markers;
coordinates and cell lengths in angstrom; the time step in AKMA units
(dt / 0.04888821 ps); the cell record as [a, cos gamma, b, cos beta,
cos alpha, c] from the edge lengths and the dot-product ratios of the box
vectors; the frame count (NSET) and last step (NSTEP) patched into the header
once known.  The log is OpenMM's `StateDataReporter` CSV for the flags the
protocol passes, whose column order is OpenMM's fixed one, `--` for the first
row's speed.
"""

from __future__ import annotations

import struct
from typing import BinaryIO, Optional, Sequence

import numpy as np

from .system import State, serialise_state

AKMA_PICOSECONDS = 0.04888821
DCD_HEADER_BYTES = 276
_NSET_OFFSET, _NSTEP_OFFSET = 8, 20

LOG_COLUMNS = ("Step", "Potential Energy (kJ/mole)", "Kinetic Energy (kJ/mole)", "Total Energy (kJ/mole)",
               "Temperature (K)", "Box Volume (nm^3)", "Speed (ns/day)")


def unit_cell(box) -> tuple:
    """Edge lengths (nm) and the cosines (cos alpha, cos beta, cos gamma) of
    three box vectors: alpha between b and c, beta between a and c, gamma
    between a and b."""
    a, b, c = np.asarray(box, dtype=np.float64).reshape(3, 3)
    la, lb, lc = (float(np.sqrt(v @ v)) for v in (a, b, c))
    return (la, lb, lc), (float(b @ c) / (lb * lc), float(a @ c) / (la * lc), float(a @ b) / (la * lb))


class DcdWriter:
    """`DcdWriter`, src/analysis/dcd.ts: header, frames, then the header patch.
    With a seekable `stream` (a file opened "w+b"), `write_frame` keeps NSET and
    NSTEP current, as OpenMM does after every frame."""

    def __init__(self, stream: BinaryIO, particle_count: int, time_step: float, first_step: int = 0,
                 interval: int = 1, periodic: bool = True, titles: Optional[Sequence[str]] = None):
        if particle_count <= 0:
            raise ValueError(f"a DCD needs at least one particle, got {particle_count}")
        self.stream = stream
        self.n = int(particle_count)
        self.first_step = int(first_step)
        self.interval = int(interval)
        self.periodic = bool(periodic)
        self.frames = 0
        self.stream.write(self._header(time_step, titles or ("Created by making-it-rain-webgpu_b200",)))

    def _header(self, time_step: float, titles: Sequence[str]) -> bytes:
        icntrl = [0, self.first_step, self.interval, 0, 0, 0, 0, 0, 0]
        head = struct.pack("<i4s9if10i", 84, b"CORD", *icntrl, time_step / AKMA_PICOSECONDS,
                           1 if self.periodic else 0, 0, 0, 0, 0, 0, 0, 0, 0, 24)
        head += struct.pack("<i", 84)
        lines = [(titles[k] if k < len(titles) else "").encode("ascii", "replace")[:80] for k in range(2)]
        head += struct.pack("<ii80s80si", 164, 2, lines[0], lines[1], 164)
        head += struct.pack("<iii", 4, self.n, 4)
        assert len(head) == DCD_HEADER_BYTES
        return head

    @property
    def frame_bytes(self) -> int:
        return 3 * (8 + 4 * self.n) + (56 if self.periodic else 0)

    def write_frame(self, positions, box=None) -> None:
        """One frame: positions (N, 3) nm; `box` the three cell vectors (nm),
        required when the file is periodic."""
        p = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
        if p.shape[0] != self.n:
            raise ValueError(f"expected {self.n} particles, got {p.shape[0]}")
        if not np.all(np.isfinite(p)):
            raise ValueError("a non-finite coordinate: refusing to write it into the trajectory")
        out = b""
        if self.periodic:
            if box is None:
                raise ValueError("a periodic DCD needs the cell of every frame")
            (la, lb, lc), (ca, cb, cg) = unit_cell(box)
            out += struct.pack("<i6di", 48, 10 * la, cg, 10 * lb, cb, ca, 10 * lc, 48)
        for axis in range(3):
            out += struct.pack("<i", 4 * self.n) + (10.0 * p[:, axis]).astype("<f4").tobytes() + \
                struct.pack("<i", 4 * self.n)
        self.stream.write(out)
        self.frames += 1
        if self.stream.seekable():
            end = self.stream.tell()
            for offset, value in self.header_patches():
                self.stream.seek(offset)
                self.stream.write(struct.pack("<i", value))
            self.stream.seek(end)

    def header_patches(self):
        """(offset, value) of the two header words that depend on the frames written."""
        return [(_NSET_OFFSET, self.frames),
                (_NSTEP_OFFSET, self.first_step + max(0, self.frames - 1) * self.interval)]


def read_dcd(data: bytes) -> dict:
    """The header fields, cells and coordinates (nm) of a DCD this module wrote."""
    marker, tag = struct.unpack_from("<i4s", data, 0)
    if marker != 84 or tag != b"CORD":
        raise ValueError("not a CHARMM DCD")
    icntrl = struct.unpack_from("<9if10i", data, 8)
    nset, istart, nsavc, nstep = icntrl[0], icntrl[1], icntrl[2], icntrl[3]
    delta, periodic = icntrl[9], icntrl[10] == 1
    n = struct.unpack_from("<i", data, DCD_HEADER_BYTES - 8)[0]
    at = DCD_HEADER_BYTES
    cells, coords = [], []
    for _ in range(nset):
        if periodic:
            cells.append(struct.unpack_from("<6d", data, at + 4))
            at += 56
        xyz = []
        for _axis in range(3):
            xyz.append(np.frombuffer(data, dtype="<f4", count=n, offset=at + 4).astype(np.float64) / 10.0)
            at += 8 + 4 * n
        coords.append(np.stack(xyz, axis=1))
    return {"frames": nset, "first_step": istart, "interval": nsavc, "last_step": nstep,
            "time_step": delta * AKMA_PICOSECONDS, "periodic": periodic, "atoms": n, "cells": cells,
            "positions": coords}


def log_header() -> str:
    """OpenMM's StateDataReporter header line for the protocol's flags."""
    return "#" + ",".join(f'"{c}"' for c in LOG_COLUMNS) + "\n"


def log_row(step: int, potential: float, kinetic: float, temperature: float, volume: float,
            speed: Optional[float]) -> str:
    """One log row; the total is potential + kinetic; `speed` None on the first row."""
    values = [str(int(step)), repr(float(potential)), repr(float(kinetic)), repr(float(potential + kinetic)),
              repr(float(temperature)), repr(float(volume)), "--" if speed is None else repr(float(speed))]
    return ",".join(values) + "\n"


def checkpoint(loop, system: int = 0, time_step: Optional[float] = None) -> str:
    """The `.rst` State XML of one system of a running engine (positions,
    velocities, box, step, time), which `parse_state` and OpenMM read back."""
    dt = time_step if time_step is not None else loop.options.time_step
    step = loop.steps
    return serialise_state(State(positions=loop.positions(system), box=loop.box_vectors(system),
                                 velocities=loop.velocities(system), step=step, time=step * dt))
