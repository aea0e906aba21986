"""Minimal Exodus II writer in the netCDF classic encodings (test infrastructure: it makes
the mesh files the reader in platoanalyze_b200/csrc/exodus.cpp is tested on).

write_exodus(path, coords, conn, node_sets, side_sets, version=2)
  coords (N,3) float64, conn (C,4) 0-based int; node_sets {name: 0-based nodes};
  side_sets {name: (0-based cells, 1-based Exodus side numbers)}; version 1 (CDF-1, 32-bit
  offsets), 2 (CDF-2, 64-bit offsets) or 5 (CDF-5, 64-bit data, int64 connectivity).
Run as a script to (re)make tests/decks/box_6x3x3.exo.
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

NC_CHAR, NC_INT, NC_DOUBLE, NC_INT64 = 2, 4, 6, 10
SIZES = {NC_CHAR: 1, NC_INT: 4, NC_DOUBLE: 8, NC_INT64: 8}
LEN_NAME = 33


def _pad(b: bytes) -> bytes:
    return b + b"\0" * ((4 - len(b) % 4) % 4)


def write_exodus(path, coords, conn, node_sets: dict, side_sets: dict, version: int = 2) -> None:
    coords = np.asarray(coords, np.float64)
    conn = np.asarray(conn, np.int64)
    big = version == 5
    itype = NC_INT64 if big else NC_INT

    def cnt(n):  # counts and dimension lengths
        return struct.pack(">Q", n) if big else struct.pack(">I", n)

    def name(s):
        b = s.encode()
        return cnt(len(b)) + _pad(b)

    dims = [("len_name", LEN_NAME), ("four", 4), ("num_dim", 3), ("num_nodes", len(coords)), ("num_elem", len(conn)),
            ("num_el_blk", 1), ("num_el_in_blk1", len(conn)), ("num_nod_per_el1", 4)]
    if node_sets:
        dims.append(("num_node_sets", len(node_sets)))
    if side_sets:
        dims.append(("num_side_sets", len(side_sets)))
    for k, nodes in enumerate(node_sets.values(), 1):
        dims.append((f"num_nod_ns{k}", len(nodes)))
    for k, (cells, _) in enumerate(side_sets.values(), 1):
        dims.append((f"num_side_ss{k}", len(cells)))
    dims.append(("time_step", 0))  # the record dimension (no records written)
    did = {n: i for i, (n, _) in enumerate(dims)}

    def names_table(keys):
        a = np.zeros((len(keys), LEN_NAME), np.uint8)
        for i, k in enumerate(keys):
            b = k.encode()[:LEN_NAME - 1]
            a[i, :len(b)] = list(b)
        return a.tobytes()

    def ints(a):
        a = np.asarray(a, np.int64)
        return a.astype(">i8").tobytes() if big else a.astype(">i4").tobytes()

    # (name, dim names, type, data bytes, text attributes)
    vars_ = [(f"coord{c}", ["num_nodes"], NC_DOUBLE, coords[:, i].astype(">f8").tobytes(), {})
             for i, c in enumerate("xyz")]
    vars_.append(("connect1", ["num_el_in_blk1", "num_nod_per_el1"], itype, ints(conn + 1), {"elem_type": "TETRA"}))
    vars_.append(("eb_prop1", ["num_el_blk"], NC_INT, np.array([1], ">i4").tobytes(), {"name": "ID"}))
    if node_sets:
        vars_.append(("ns_prop1", ["num_node_sets"], NC_INT, np.arange(1, len(node_sets) + 1, dtype=">i4").tobytes(),
                      {"name": "ID"}))
        vars_.append(("ns_names", ["num_node_sets", "len_name"], NC_CHAR, names_table(list(node_sets)), {}))
        for k, nodes in enumerate(node_sets.values(), 1):
            vars_.append((f"node_ns{k}", [f"num_nod_ns{k}"], itype, ints(np.asarray(nodes) + 1), {}))
    if side_sets:
        vars_.append(("ss_prop1", ["num_side_sets"], NC_INT, np.arange(1, len(side_sets) + 1, dtype=">i4").tobytes(),
                      {"name": "ID"}))
        vars_.append(("ss_names", ["num_side_sets", "len_name"], NC_CHAR, names_table(list(side_sets)), {}))
        for k, (cells, sides) in enumerate(side_sets.values(), 1):
            vars_.append((f"elem_ss{k}", [f"num_side_ss{k}"], itype, ints(np.asarray(cells) + 1), {}))
            vars_.append((f"side_ss{k}", [f"num_side_ss{k}"], itype, ints(sides), {}))

    def header(begins):
        h = b"CDF" + bytes([version]) + cnt(0)
        h += struct.pack(">I", 0x0A) + cnt(len(dims))
        for n, l in dims:
            h += name(n) + cnt(l)
        h += struct.pack(">I", 0x0C) + cnt(1)  # one global attribute
        h += name("title") + struct.pack(">I", NC_CHAR) + cnt(len(b"b200 test mesh")) + _pad(b"b200 test mesh")
        h += struct.pack(">I", 0x0B) + cnt(len(vars_))
        for (n, dn, t, data, att), b in zip(vars_, begins):
            h += name(n) + cnt(len(dn)) + b"".join(cnt(did[d]) for d in dn)
            if att:
                h += struct.pack(">I", 0x0C) + cnt(len(att))
                for an, av in att.items():
                    ab = av.encode()
                    h += name(an) + struct.pack(">I", NC_CHAR) + cnt(len(ab)) + _pad(ab)
            else:
                h += struct.pack(">I", 0) + cnt(0)
            vsize = len(_pad(data))
            h += struct.pack(">I", t) + cnt(vsize)
            h += struct.pack(">I", b) if version == 1 else struct.pack(">Q", b)
        return h

    hlen = len(header([0] * len(vars_)))
    begins, off = [], hlen
    for v in vars_:
        begins.append(off)
        off += len(_pad(v[3]))
    out = header(begins) + b"".join(_pad(v[3]) for v in vars_)
    Path(path).write_bytes(out)


def box_sets(m):
    """x-, x+, y-, y+, z-, z+ node and side sets of a generated box mesh (Exodus side numbers)."""
    from platoanalyze_b200.mesh import TET_FACES

    names = ["x-", "x+", "y-", "y+", "z-", "z+"]
    ns = {n: m.nodeset(f) for f, n in enumerate(names)}
    ss = {}
    for f, n in enumerate(names):
        cells, local = m.sideset(f)
        sides = []
        for lc in local:
            key = sorted(lc.tolist())
            sides.append(1 + next(i for i, t in enumerate(TET_FACES) if sorted(t.tolist()) == key))
        ss[n] = (cells, np.array(sides))
    return ns, ss


if __name__ == "__main__":
    import sys

    sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
    from platoanalyze_b200.mesh import box_mesh

    m = box_mesh(6, 3, 3, 2.0, 1.0, 1.0)
    ns, ss = box_sets(m)
    out = Path(__file__).resolve().parents[1] / "decks" / "box_6x3x3.exo"
    write_exodus(out, m.coords, m.connectivity, ns, ss, version=2)
    print(out, out.stat().st_size, "bytes")
