"""Space-group operations for the oracle, generated from Hall symbols.

TEST INFRASTRUCTURE ONLY.  The reference takes its operations from Crystalline.jl
(`operations(spacegroup(sg, dim))`, src/symmetry_ops.jl:51-53), which is not
vendored in the reference tree.  The oracle needs an operation source of its own,
independent of the library under test (whose table, csrc/spacegroups.cpp, closes
ITA general-position generators).  This module uses a different, published
encoding: the explicit-origin space-group notation of S. R. Hall, Acta Cryst. A37,
517-525 (1981), one Hall symbol per group in the ITA standard setting (monoclinic
unique axis b, cell choice 1; origin choice 2 where ITA gives two; hexagonal axes,
obverse centring, for the rhombohedral groups).

A Hall symbol is  L [N^A_T]... (V):
  L     lattice letter (P A B C I R F), preceded by '-' for a centre of symmetry at
        the origin;
  N     rotation order 1 2 3 4 6, preceded by '-' for the improper rotation;
  A     axis x y z, ' or " (face diagonals, relative to the preceding axis), * (the
        body diagonal); omitted axes follow Hall's default rules;
  T     translation letters a b c n u v w d, or a screw digit (k/N along the axis);
  V     origin shift in twelfths: (R, t) -> (R, t + (I - R) V).
The group is the closure of the generators and the centring translations modulo
integer lattice translations.  Plane groups use the same notation restricted to
the (x, y) block of the 3-D symbols of their layer equivalents.

get_ops follows convert_op (src/symmetry_ops.jl:38-46): fractional translations in
[0, 1) times N, required to be integral.
"""
from __future__ import annotations

from fractions import Fraction

import numpy as np

DEN = 12  # every translation here is a multiple of 1/12

HALL_3D = {
    1: "P 1", 2: "-P 1", 3: "P 2y", 4: "P 2yb", 5: "C 2y", 6: "P -2y", 7: "P -2yc", 8: "C -2y", 9: "C -2yc",
    10: "-P 2y", 11: "-P 2yb", 12: "-C 2y", 13: "-P 2yc", 14: "-P 2ybc", 15: "-C 2yc",
    16: "P 2 2", 17: "P 2c 2", 18: "P 2 2ab", 19: "P 2ac 2ab", 20: "C 2c 2", 21: "C 2 2", 22: "F 2 2",
    23: "I 2 2", 24: "I 2b 2c", 25: "P 2 -2", 26: "P 2c -2", 27: "P 2 -2c", 28: "P 2 -2a", 29: "P 2c -2ac",
    30: "P 2 -2bc", 31: "P 2ac -2", 32: "P 2 -2ab", 33: "P 2c -2n", 34: "P 2 -2n", 35: "C 2 -2", 36: "C 2c -2",
    37: "C 2 -2c", 38: "A 2 -2", 39: "A 2 -2c", 40: "A 2 -2a", 41: "A 2 -2ac", 42: "F 2 -2", 43: "F 2 -2d",
    44: "I 2 -2", 45: "I 2 -2c", 46: "I 2 -2a", 47: "-P 2 2", 48: "-P 2ab 2bc", 49: "-P 2 2c", 50: "-P 2ab 2b",
    51: "-P 2a 2a", 52: "-P 2a 2bc", 53: "-P 2ac 2", 54: "-P 2a 2ac", 55: "-P 2 2ab", 56: "-P 2ab 2ac",
    57: "-P 2c 2b", 58: "-P 2 2n", 59: "-P 2ab 2a", 60: "-P 2n 2ab", 61: "-P 2ac 2ab", 62: "-P 2ac 2n",
    63: "-C 2c 2", 64: "-C 2bc 2", 65: "-C 2 2", 66: "-C 2 2c", 67: "-C 2b 2", 68: "-C 2b 2bc", 69: "-F 2 2",
    70: "-F 2uv 2vw", 71: "-I 2 2", 72: "-I 2 2c", 73: "-I 2b 2c", 74: "-I 2b 2",
    75: "P 4", 76: "P 4w", 77: "P 4c", 78: "P 4cw", 79: "I 4", 80: "I 4bw", 81: "P -4", 82: "I -4", 83: "-P 4",
    84: "-P 4c", 85: "-P 4a", 86: "-P 4bc", 87: "-I 4", 88: "-I 4ad", 89: "P 4 2", 90: "P 4ab 2ab", 91: "P 4w 2c",
    92: "P 4abw 2nw", 93: "P 4c 2", 94: "P 4n 2n", 95: "P 4cw 2c", 96: "P 4nw 2abw", 97: "I 4 2", 98: "I 4bw 2bw",
    99: "P 4 -2", 100: "P 4 -2ab", 101: "P 4c -2c", 102: "P 4n -2n", 103: "P 4 -2c", 104: "P 4 -2n",
    105: "P 4c -2", 106: "P 4c -2ab", 107: "I 4 -2", 108: "I 4 -2c", 109: "I 4bw -2", 110: "I 4bw -2c",
    111: "P -4 2", 112: "P -4 2c", 113: "P -4 2ab", 114: "P -4 2n", 115: "P -4 -2", 116: "P -4 -2c",
    117: "P -4 -2ab", 118: "P -4 -2n", 119: "I -4 -2", 120: "I -4 -2c", 121: "I -4 2", 122: "I -4 2bw",
    123: "-P 4 2", 124: "-P 4 2c", 125: "-P 4a 2b", 126: "-P 4a 2bc", 127: "-P 4 2ab", 128: "-P 4 2n",
    129: "-P 4a 2a", 130: "-P 4a 2ac", 131: "-P 4c 2", 132: "-P 4c 2c", 133: "-P 4ac 2b", 134: "-P 4ac 2bc",
    135: "-P 4c 2ab", 136: "-P 4n 2n", 137: "-P 4ac 2a", 138: "-P 4ac 2ac", 139: "-I 4 2", 140: "-I 4 2c",
    141: "-I 4bd 2", 142: "-I 4bd 2c",
    143: "P 3", 144: "P 31", 145: "P 32", 146: "R 3", 147: "-P 3", 148: "-R 3", 149: "P 3 2", 150: 'P 3 2"',
    151: "P 31 2c (0 0 1)", 152: 'P 31 2"', 153: "P 32 2c (0 0 -1)", 154: 'P 32 2"', 155: 'R 3 2"',
    156: 'P 3 -2"', 157: "P 3 -2", 158: 'P 3 -2"c', 159: "P 3 -2c", 160: 'R 3 -2"', 161: 'R 3 -2"c',
    162: "-P 3 2", 163: "-P 3 2c", 164: '-P 3 2"', 165: '-P 3 2"c', 166: '-R 3 2"', 167: '-R 3 2"c',
    168: "P 6", 169: "P 61", 170: "P 65", 171: "P 62", 172: "P 64", 173: "P 6c", 174: "P -6", 175: "-P 6",
    176: "-P 6c", 177: "P 6 2", 178: "P 61 2 (0 0 -1)", 179: "P 65 2 (0 0 1)", 180: "P 62 2c (0 0 1)",
    181: "P 64 2c (0 0 -1)", 182: "P 6c 2c", 183: "P 6 -2", 184: "P 6 -2c", 185: "P 6c -2", 186: "P 6c -2c",
    187: "P -6 2", 188: "P -6c 2", 189: "P -6 -2", 190: "P -6c -2c", 191: "-P 6 2", 192: "-P 6 2c",
    193: "-P 6c 2", 194: "-P 6c 2c",
    195: "P 2 2 3", 196: "F 2 2 3", 197: "I 2 2 3", 198: "P 2ac 2ab 3", 199: "I 2b 2c 3", 200: "-P 2 2 3",
    201: "-P 2ab 2bc 3", 202: "-F 2 2 3", 203: "-F 2uv 2vw 3", 204: "-I 2 2 3", 205: "-P 2ac 2ab 3",
    206: "-I 2b 2c 3", 207: "P 4 2 3", 208: "P 4n 2 3", 209: "F 4 2 3", 210: "F 4d 2 3", 211: "I 4 2 3",
    212: "P 4acd 2ab 3", 213: "P 4bd 2ab 3", 214: "I 4bd 2c 3", 215: "P -4 2 3", 216: "F -4 2 3",
    217: "I -4 2 3", 218: "P -4n 2 3", 219: "F -4c 2 3", 220: "I -4bd 2c 3", 221: "-P 4 2 3",
    222: "-P 4a 2bc 3", 223: "-P 4n 2 3", 224: "-P 4bc 2bc 3", 225: "-F 4 2 3", 226: "-F 4c 2 3",
    227: "-F 4vw 2vw 3", 228: "-F 4cvw 2vw 3", 229: "-I 4 2 3", 230: "-I 4bd 2c 3",
}

# Plane groups: the 3-D symbol of the layer group with the same (x, y) action.
HALL_2D = {
    1: "P 1", 2: "P 2", 3: "P -2x", 4: "P -2xb", 5: "C -2x", 6: "P 2 -2", 7: "P 2 -2a", 8: "P 2 -2ab",
    9: "C 2 -2", 10: "P 4", 11: "P 4 -2", 12: "P 4 -2ab", 13: "P 3", 14: 'P 3 -2"', 15: "P 3 -2", 16: "P 6",
    17: "P 6 -2",
}

_LATTICE = {
    "P": [],
    "A": [(0, 6, 6)],
    "B": [(6, 0, 6)],
    "C": [(6, 6, 0)],
    "I": [(6, 6, 6)],
    "R": [(8, 4, 4), (4, 8, 8)],
    "F": [(0, 6, 6), (6, 0, 6), (6, 6, 0)],
}

_TRANS = {"a": (6, 0, 0), "b": (0, 6, 0), "c": (0, 0, 6), "n": (6, 6, 6), "u": (3, 0, 0), "v": (0, 3, 0),
          "w": (0, 0, 3), "d": (3, 3, 3)}

# Proper rotations about the principal axes (Hall 1981, Table 3).
_ROT = {
    ("x", 2): [[1, 0, 0], [0, -1, 0], [0, 0, -1]],
    ("x", 3): [[1, 0, 0], [0, 0, -1], [0, 1, -1]],
    ("x", 4): [[1, 0, 0], [0, 0, -1], [0, 1, 0]],
    ("x", 6): [[1, 0, 0], [0, 1, -1], [0, 1, 0]],
    ("y", 2): [[-1, 0, 0], [0, 1, 0], [0, 0, -1]],
    ("y", 3): [[-1, 0, 1], [0, 1, 0], [-1, 0, 0]],
    ("y", 4): [[0, 0, 1], [0, 1, 0], [-1, 0, 0]],
    ("y", 6): [[0, 0, 1], [0, 1, 0], [-1, 0, 1]],
    ("z", 2): [[-1, 0, 0], [0, -1, 0], [0, 0, 1]],
    ("z", 3): [[0, -1, 0], [1, -1, 0], [0, 0, 1]],
    ("z", 4): [[0, -1, 0], [1, 0, 0], [0, 0, 1]],
    ("z", 6): [[1, -1, 0], [1, 0, 0], [0, 0, 1]],
}
# Two-fold rotations about face diagonals, keyed by the preceding axis: ' and ".
_DIAG2 = {
    ("x", "'"): [[-1, 0, 0], [0, 0, -1], [0, -1, 0]],
    ("x", '"'): [[-1, 0, 0], [0, 0, 1], [0, 1, 0]],
    ("y", "'"): [[0, 0, -1], [0, -1, 0], [-1, 0, 0]],
    ("y", '"'): [[0, 0, 1], [0, -1, 0], [1, 0, 0]],
    ("z", "'"): [[0, -1, 0], [-1, 0, 0], [0, 0, -1]],
    ("z", '"'): [[0, 1, 0], [1, 0, 0], [0, 0, -1]],
}
_BODY3 = [[0, 0, 1], [1, 0, 0], [0, 1, 0]]
_AXIS_INDEX = {"x": 0, "y": 1, "z": 2}


def _tokens(symbol):
    """Split a Hall symbol into its lattice part, rotation parts and origin shift."""
    s = symbol.strip()
    shift = (0, 0, 0)
    if "(" in s:
        s, v = s.split("(")
        shift = tuple(int(x) for x in v.rstrip(")").split())
    parts = s.split()
    return parts[0], parts[1:], shift


def _parse_rotation(tok, k, prev_order, prev_axis):
    """One matrix symbol -> (R, t numerators over DEN, order, axis)."""
    improper = tok.startswith("-")
    if improper:
        tok = tok[1:]
    order = int(tok[0])
    rest = tok[1:]
    axis = None
    if rest and rest[0] in "xyz'\"*":
        axis, rest = rest[0], rest[1:]
    screw = 0
    if rest and rest[0].isdigit():
        screw, rest = int(rest[0]), rest[1:]
    if axis is None:  # Hall's default axis rules
        if k == 0:
            axis = "z"
        elif k == 1 and order == 2:
            axis = "x" if prev_order in (2, 4) else "'"
        elif order == 3:
            axis = "*"
        else:
            raise ValueError(f"no default axis for {tok!r} at position {k}")
    if order == 1:
        R = np.eye(3, dtype=np.int64)
    elif axis in _AXIS_INDEX:
        R = np.array(_ROT[(axis, order)], dtype=np.int64)
    elif axis in ("'", '"'):
        if order != 2:
            raise ValueError(tok)
        R = np.array(_DIAG2[(prev_axis, axis)], dtype=np.int64)
    else:  # body diagonal
        if order != 3:
            raise ValueError(tok)
        R = np.array(_BODY3, dtype=np.int64)
    t = np.zeros(3, dtype=np.int64)
    if screw:
        if axis not in _AXIS_INDEX:
            raise ValueError(f"screw on a non-principal axis: {tok!r}")
        t[_AXIS_INDEX[axis]] += DEN * screw // order
    for ch in rest:
        t += np.array(_TRANS[ch], dtype=np.int64)
    if improper:
        R = -R
    return R, t, order, axis if axis in _AXIS_INDEX else prev_axis


def _closure(gens):
    """All products of the generators, modulo integer translations (numerators mod DEN)."""
    key = lambda R, t: (tuple(R.ravel().tolist()), tuple((t % DEN).tolist()))
    ident = (np.eye(3, dtype=np.int64), np.zeros(3, dtype=np.int64))
    elems = {key(*ident): ident}
    frontier = [ident]
    while frontier:
        new = []
        for R1, t1 in frontier:
            for R2, t2 in gens:
                R, t = R1 @ R2, (R1 @ t2 + t1) % DEN
                k = key(R, t)
                if k not in elems:
                    elems[k] = (R, t)
                    new.append((R, t))
        frontier = new
    return list(elems.values())


def hall_ops(symbol):
    """Fractional operations of a Hall symbol: list of (R 3x3 int, t int numerators / DEN in [0, DEN))."""
    lat, rots, V = _tokens(symbol)
    centro = lat.startswith("-")
    lat = lat.lstrip("-")
    gens = []
    prev_order, prev_axis = None, "z"
    for k, tok in enumerate(rots):
        R, t, prev_order, prev_axis = _parse_rotation(tok, k, prev_order, prev_axis)
        gens.append((R, t))
    if centro:
        gens.append((-np.eye(3, dtype=np.int64), np.zeros(3, dtype=np.int64)))
    Vv = np.array(V, dtype=np.int64)
    gens = [(R, (t + (np.eye(3, dtype=np.int64) - R) @ Vv) % DEN) for R, t in gens]
    for c in _LATTICE[lat]:
        gens.append((np.eye(3, dtype=np.int64), np.array(c, dtype=np.int64)))
    ops = _closure(gens)
    # identity first, then by rotation and translation (a fixed, documented order)
    ops.sort(key=lambda o: (not (np.array_equal(o[0], np.eye(3, dtype=np.int64)) and not o[1].any()),
                            tuple(-o[0].ravel()), tuple(o[1])))
    return ops


def fractional_ops(sg, dim=3):
    """Operations of space group `sg` (plane group for dim = 2) as (R, t) with t a tuple
    of Fractions in [0, 1)."""
    table = HALL_3D if dim == 3 else HALL_2D
    if sg not in table:
        raise KeyError(f"no Hall symbol for group {sg} in {dim}-D")
    out, seen = [], set()
    for R, t in hall_ops(table[sg]):
        Rd = R[:dim, :dim]
        td = t[:dim]
        if dim == 2 and (R[2, 2] != 1 or R[0, 2] or R[1, 2] or R[2, 0] or R[2, 1]):
            continue  # operations that flip z have no plane-group counterpart
        k = (tuple(Rd.ravel().tolist()), tuple(td.tolist()))
        if k in seen:
            continue
        seen.add(k)
        out.append((Rd.copy(), tuple(Fraction(int(v), DEN) for v in td)))
    return out


def get_ops(sg, dim, N, SymOp):
    """get_ops (src/symmetry_ops.jl:51-53) with convert_op (:38-46): grid-unit operations,
    `SymOp(R_tuple, t_tuple)` built by the caller's class."""
    out = []
    for R, t in fractional_ops(sg, dim):
        tg = []
        for d in range(dim):
            v = t[d] * N[d]
            if v.denominator != 1:
                raise ValueError(f"Symmetry operation not commensurate with grid {tuple(N)}")
            tg.append(int(v))
        out.append(SymOp(tuple(int(x) for x in R.ravel()), tuple(tg)))
    return out
