"""Mesh descriptors: the product builder against the oracle's restatement of
DSEM's setup, and the 22^3 topology against the reference's shipped files."""
import os

import numpy as np
import pytest

from dsem_b200 import mesh

# The reference checkout's 22^3 case folder (p8-22x22x22) is read only when
# DSEM_REFERENCE_DIR names the checkout; the tests that need it skip otherwise.
REF = os.path.join(os.environ.get("DSEM_REFERENCE_DIR", ""), "p8-22x22x22") \
    if os.environ.get("DSEM_REFERENCE_DIR") else ""
KEYS = ("ncg", "jacob", "gmetg", "gmet", "mortar", "n_hat", "norm")


@pytest.mark.parametrize("n,p,rot", [(4, 4, None), (3, 2, {13: 5}), (3, 6, {13: 22}), (2, 3, None)])
def test_builder_matches_oracle_bitwise(oracle_mod, n, p, rot):
    r = None
    if rot:
        r = [0] * n ** 3
        for k, v in rot.items():
            r[k] = v
    b = mesh.Box(n, n, n, p, rot=r)
    d = b.desc()
    od = oracle_mod.Case.box(n, n, n, p, rot=r).export_desc(b.ldx)
    for k in KEYS:
        assert np.array_equal(d[k], od[k]), k


def test_mixed_order_band(oracle_mod):
    """p-nonconforming band (middle third in x at p = 8 inside p = 6)."""
    n = 3
    orders = np.full(n ** 3, 6)
    for iz in range(n):
        for ix in range(n):
            for iy in range(n):
                if ix == 1:
                    orders[iy + n * (ix + n * iz)] = 8
    b = mesh.Box(n, n, n, orders)
    d = b.desc()
    od = oracle_mod.Case.box(n, n, n, orders).export_desc(b.ldx)
    for k in KEYS:
        assert np.array_equal(d[k], od[k]), k
    conf = b.mortar[:, 13:17].all(axis=1)
    assert (~conf).sum() == 2 * n * n  # two faces of the band per (y, z) column
    assert set(b.mortar[~conf, 8]) == {9}


def test_tgv_22_topology(box22):
    """31,944 interface mortars after periodic pairing (DNS-22p8.graph header 10648 31944)."""
    b = box22
    assert b.nel == 10648 and b.nmort == 31944
    assert set(b.mortar[:, 10]) == {0} and set(b.mortar[:, 11]) == {1} and set(b.mortar[:, 12]) == {1}
    if os.path.exists(os.path.join(REF, "DNS-22p8.graph")):
        with open(os.path.join(REF, "DNS-22p8.graph")) as f:
            ne, nm = (int(x) for x in f.readline().split()[:2])
        assert (ne, nm) == (10648, 31944)
        # element adjacency equals the METIS graph shipped with the reference,
        # except that the shipped file lists an element on the x = 0 / x = 2pi
        # boundary as its own x-periodic neighbour (a partitioning-file quirk;
        # the mortars themselves pair the two elements)
        adj = [set() for _ in range(b.nel)]
        for m in b.mortar:
            adj[m[0] - 1].add(int(m[1]))
            adj[m[1] - 1].add(int(m[0]))
        xper = {}
        for m in b.mortar:
            if (m[2], m[3]) == (4, 6):
                xper[m[0] - 1] = int(m[1])
                xper[m[1] - 1] = int(m[0])
        with open(os.path.join(REF, "DNS-22p8.graph")) as f:
            f.readline()
            for e in range(b.nel):
                ref = set(int(x) for x in f.readline().split())
                assert adj[e] - ref <= {xper.get(e)}
                assert ref - adj[e] <= {e + 1}


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "tgv-22x22x22-p8.mesh")), reason="reference mesh absent")
def test_shipped_mesh_nodes_match(box22):
    """The generated element corners equal the shipped mesh's to its printed precision."""
    b = box22
    nodes = {}
    elems = []
    with open(os.path.join(REF, "tgv-22x22x22-p8.mesh")) as f:
        lines = f.read().splitlines()
    i = lines.index("nodes") + 1
    while not lines[i].startswith("end"):
        t = lines[i].split()
        nodes[int(t[0])] = np.array([float(x) for x in t[1:4]])
        i += 1
    i = lines.index("elements") + 1
    while not lines[i].startswith("end"):
        hdr = lines[i].split()
        conn = [int(x) for x in lines[i + 1].split()]
        elems.append((int(hdr[0]), conn))
        i += 2
    assert len(elems) == 10648
    for eid, conn in elems[::97]:
        corners = np.array([nodes[k] for k in conn])
        assert np.abs(corners - b.corner[eid - 1]).max() <= 1e-12


def test_tgv_22_against_shipped_files_fixture(box22):
    """The 22^3 mesh builder against the reference's shipped files through
    tests/golden/mesh_22cube_p8.json (tests/golden/make_mesh_fixture.py wrote it from
    DNS-22p8.graph and tgv-22x22x22-p8.mesh): the graph's header, every element's neighbour
    list (a SHA-256 of the sorted lists), and the corners of a sample of elements to the mesh
    file's printed precision.  The shipped graph lists each element of the x = 0 layer as its
    own neighbour in place of its x-periodic neighbour on the x = 2 pi layer (a partitioning
    file quirk; the mortars pair the two elements), so the builder's lists take the same
    form before hashing."""
    import json
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_mesh_fixture import adjacency_digest
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mesh_22cube_p8.json")) as f:
        fx = json.load(f)
    n = 22
    b = box22
    assert [b.nel, b.nmort] == fx["graph_header"] and fx["elements_in_mesh_file"] == b.nel
    adj = [set() for _ in range(b.nel)]
    for m in b.mortar:
        adj[m[0] - 1].add(int(m[1]))
        adj[m[1] - 1].add(int(m[0]))
    ix = lambda e: (e // n) % n  # element e = iy + n (ix + n iz), 0-based
    self_listed = set(fx["self_listed"])
    assert self_listed == {e + 1 for e in range(b.nel) if ix(e) == 0}
    for e1 in self_listed:
        e = e1 - 1
        wrap = [nb for nb in adj[e] if abs(ix(nb - 1) - ix(e)) == n - 1]
        assert len(wrap) == 1
        adj[e].discard(wrap[0])
        adj[e].add(e1)
    assert adjacency_digest(adj) == fx["adjacency_sha256"]
    for eid, corners in fx["corner_sample"].items():
        assert np.abs(np.array(corners) - b.corner[int(eid) - 1]).max() <= 1e-12, eid
