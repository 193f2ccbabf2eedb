"""``.in`` parsing, depth interpolation and PETSc-binary vectors (oracle; test infrastructure only).

Restates the key/value loop that every reference class repeats
(e.g. source/domain.cpp:133-196), ``loadVectorFromInputFile``
(source/genFuncs.cpp:413-440 for numbers, :476-505 for strings), ``setVec``
(source/genFuncs.cpp:574-617) and the PETSc binary Vec format read by
``loadVecFromInputFile`` (source/genFuncs.cpp:380-410) and documented by
matlab/visualizePetsc/loadVec.m:45-78 (big-endian int32 class id 1211214,
int32 length, big-endian float64 payload, records appended back to back).
"""
import re
import struct

import numpy as np

DELIM = " = "
VEC_FILE_CLASSID = 1211214
NPOS = (1 << 64) - 1  # std::string::npos


def _find(s, sub):
    i = s.find(sub)
    return NPOS if i < 0 else i


def _substr(s, pos, count=NPOS):
    # std::string::substr semantics with size_t wrap-around
    pos &= NPOS
    if pos > len(s):
        raise IndexError("substr position out of range")
    return s[pos:] if count >= NPOS else s[pos:pos + count]


def parse_lines(text):
    """Yield (var, rhs, rhsFull) for each line as domain.cpp:153-166 does."""
    for line in text.split("\n"):
        pos = _find(line, DELIM)
        var = _substr(line, 0, pos)
        rhs = ""
        if len(line) > ((pos + len(DELIM)) & NPOS):
            rhs = _substr(line, pos + len(DELIM))
        rhs_full = rhs
        p = _find(rhs, " ")
        rhs = _substr(rhs, 0, p)
        yield var, rhs, rhs_full


def load_vector_double(s):
    """genFuncs.cpp:413-440.  Note a one-element list yields [] (the loop runs
    only while a space is found) and a doubled space yields a 0.0 entry."""
    out = []
    pos = _find(s, "]")
    rem = _substr(s, 1, (pos - 1) & NPOS)
    pos = _find(rem, " ")
    while pos != NPOS:
        pos = _find(rem, " ")
        out.append(atof(_substr(rem, 0, pos)))
        rem = _substr(rem, (pos + 1) & NPOS)
    return out


def load_vector_string(s):
    """genFuncs.cpp:476-505 (first element taken before the loop)."""
    out = []
    pos = _find(s, "]")
    rem = _substr(s, 1, (pos - 1) & NPOS)
    pos = _find(rem, " ")
    out.append(_substr(rem, 0, pos))
    rem = _substr(rem, (pos + 1) & NPOS)
    while pos != NPOS:
        pos = _find(rem, " ")
        out.append(_substr(rem, 0, pos))
        rem = _substr(rem, (pos + 1) & NPOS)
    return out


_NUM = re.compile(r"[+-]?((\d+\.?\d*)|(\.\d+))([eE][+-]?\d+)?")


def atof(s):
    """C atof: the longest numeric prefix after leading blanks, else 0.0."""
    m = _NUM.match(s.lstrip(" \t\n\r\f\v"))
    return float(m.group(0)) if m else 0.0


def atoi(s):
    s = s.lstrip(" \t\n\r\f\v")
    i = 0
    if i < len(s) and s[i] in "+-":
        i += 1
    j = i
    while j < len(s) and s[j].isdigit():
        j += 1
    try:
        return int(s[:j]) if j > i else 0
    except ValueError:
        return 0


def set_vec(coord, vals, depths):
    """Piecewise-linear interpolation with extrapolation past the last knot.

    genFuncs.cpp:574-617: start from vals[0]; for each segment, points inside
    [z0, z1] take the segment's line (later segments win on shared knots);
    points beyond the last knot extrapolate the last segment.  A coordinate
    vector of length 1 keeps vals[0].
    """
    coord = np.asarray(coord, dtype=np.float64)
    out = np.full(coord.shape, vals[0], dtype=np.float64)
    if coord.size == 1:
        return out
    n = len(depths)
    for j, z in enumerate(coord):
        for ind in range(n - 1):
            z0, z1 = depths[ind], depths[ind + 1]
            v0, v1 = vals[ind], vals[ind + 1]
            if z >= z0 and z <= z1:
                out[j] = (v1 - v0) / (z1 - z0) * (z - z0) + v0
            elif z > z1 and ind == n - 2:
                out[j] = (v1 - v0) / (z1 - z0) * (z - z0) + v0
    return out


def read_petsc_vecs(path):
    """All Vec records of a PETSc binary file, as float64 arrays."""
    data = open(path, "rb").read()
    out, off = [], 0
    while off + 8 <= len(data):
        cid, n = struct.unpack(">ii", data[off:off + 8])
        if cid != VEC_FILE_CLASSID:
            raise ValueError("not a PETSc Vec record (class id %d)" % cid)
        off += 8
        if off + 8 * n > len(data):
            raise ValueError("truncated PETSc Vec record")
        out.append(np.frombuffer(data[off:off + 8 * n], dtype=">f8").astype(np.float64))
        off += 8 * n
    return out


def write_petsc_vec(path, vec, append=False):
    vec = np.asarray(vec, dtype=np.float64)
    with open(path, "ab" if append else "wb") as f:
        f.write(struct.pack(">ii", VEC_FILE_CLASSID, vec.size))
        f.write(vec.astype(">f8").tobytes())
