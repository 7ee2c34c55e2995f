"""Snapshot hydro files from the device state, in the reference's format.

RamsesWriter::write_hydro (RAMSES-CPP src/io/RamsesWriter.cpp:145-226) writes
Fortran-style unformatted records (int32 length, payload, int32 length): the
header (ncpu, nvar, ndim, nlevelmax, nboundary, gamma), then for every level
and domain the pair (level, ncache) and, when the level has octs, one record
per child slot and variable holding the level's octs in list order.  The
records come from the device (rg_level_output forms the primitive values from
uold there), so a run whose state stays on the GPU writes an output without
downloading the state.  The tree files (amr_*.out*) describe the host's tree
and stay with the host application that owns it.
"""
import struct

import numpy as np


def _rec(f, payload):
    f.write(struct.pack("<i", len(payload)))
    f.write(payload)
    f.write(struct.pack("<i", len(payload)))


def write_hydro(path, ctx, ndim, nvar, nlevelmax, gamma, ncpu=1, nboundary=0):
    """hydro_XXXXX.out00001 of the context's current uold (single domain)."""
    with open(path, "wb") as f:
        for v in (ncpu, nvar, ndim, nlevelmax, nboundary):
            _rec(f, struct.pack("<i", v))
        _rec(f, struct.pack("<d", gamma))
        for il in range(1, nlevelmax + 1):
            for icpu in range(1, ncpu + nboundary + 1):
                rec = ctx.level_output(il, ndim, nvar) if icpu <= ncpu else np.zeros((1 << ndim, nvar, 0))
                ncache = rec.shape[2]
                _rec(f, struct.pack("<i", il))
                _rec(f, struct.pack("<i", ncache))
                if ncache:
                    for ic in range(1 << ndim):
                        for iv in range(nvar):
                            _rec(f, np.ascontiguousarray(rec[ic, iv]).astype("<f8").tobytes())
