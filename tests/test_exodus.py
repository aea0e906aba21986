"""Exodus II reader (netCDF classic encodings) against the generated box it was written from,
and its refusals; the application reads the same file as its "Input Mesh"."""
from pathlib import Path

import numpy as np
import pytest

from exodus_writer import box_sets, write_exodus
from platoanalyze_b200 import capi
from platoanalyze_b200.app import validate
from platoanalyze_b200.mesh import TET_FACES, box_mesh, read_exodus

DECKS = Path(__file__).resolve().parent / "decks"


def same_faces(conn, a, b):
    ka = sorted(tuple(sorted(conn[c, l])) for c, l in zip(*a))
    kb = sorted(tuple(sorted(conn[c, l])) for c, l in zip(*b))
    return ka == kb


def check_against_box(f, m):
    assert np.array_equal(f.coords, m.coords) and np.array_equal(f.connectivity, m.connectivity)
    for k, name in enumerate(["x-", "x+", "y-", "y+", "z-", "z+"]):
        assert np.array_equal(f.node_sets[name], m.nodeset(k))
        assert same_faces(m.connectivity, f.side_sets[name], m.sideset(k))


def test_committed_file_matches_the_box():
    check_against_box(read_exodus(DECKS / "box_6x3x3.exo"), box_mesh(6, 3, 3, 2.0, 1.0, 1.0))


@pytest.mark.parametrize("version", [1, 2, 5])
def test_every_classic_encoding(tmp_path, version):
    m = box_mesh(3, 2, 4, 1.0, 0.5, 2.0)
    ns, ss = box_sets(m)
    write_exodus(tmp_path / "m.exo", m.coords, m.connectivity, ns, ss, version=version)
    f = read_exodus(tmp_path / "m.exo")
    check_against_box(f, m)
    # Exodus side numbers map to the reference's local node triples
    cells, local = f.side_sets["x+"]
    assert all(any(np.array_equal(l, t) for t in TET_FACES) for l in local)


def test_refusals(tmp_path):
    with pytest.raises(capi.PlatoError) as e:
        read_exodus(tmp_path / "missing.exo")
    assert "cannot open" in str(e.value)
    (tmp_path / "h5.exo").write_bytes(b"\x89HDF\r\n\x1a\n" + b"\0" * 64)
    with pytest.raises(capi.PlatoError) as e:
        read_exodus(tmp_path / "h5.exo")
    assert "netCDF-4" in str(e.value)
    (tmp_path / "junk.exo").write_bytes(b"not a mesh at all")
    with pytest.raises(capi.PlatoError) as e:
        read_exodus(tmp_path / "junk.exo")
    assert "not a netCDF classic file" in str(e.value)
    good = (DECKS / "box_6x3x3.exo").read_bytes()
    (tmp_path / "cut.exo").write_bytes(good[:len(good) // 2])
    with pytest.raises(capi.PlatoError):
        read_exodus(tmp_path / "cut.exo")


def test_application_reads_the_file():
    deck = (DECKS / "cantilever.xml").read_text().replace("box:12,6,6:2.0,1.0,1.0", "box_6x3x3.exo")
    ops = (DECKS / "operations.xml").read_text()
    validate(deck, ops, base_dir=str(DECKS))
    with pytest.raises(capi.PlatoError) as e:
        validate(deck.replace('value="x+"', 'value="tip"'), ops, base_dir=str(DECKS))
    assert "no side set 'tip'" in str(e.value)
