"""Writes tests/golden/mesh_22cube_p8.json from the reference checkout's 22^3 Taylor-Green
case folder (p8-22x22x22): the METIS graph's header, the elements that list themselves as a
neighbour, a SHA-256 of every element's sorted neighbour list, the corner coordinates of a
sample of elements from the shipped mesh file, the shipped 100-way METIS partition
(DNS-22p8.graph.part.100, one part id per element, base64 of one byte each), and the local
index of each element on its rank from grid_distribution.dat, which DSEM's read_restart wrote
for that partition (restart.f90:486-496; its rank column equals the part file).
tests/test_mesh.py and tests/test_shard_plan.py check the mesh builder and the shard planner
against it without the checkout.

    python tests/golden/make_mesh_fixture.py <reference checkout>   (or DSEM_REFERENCE_DIR)
"""
import base64
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SAMPLE = 193  # every 193rd element of the mesh file (56 elements)


def adjacency_digest(neighbours):
    """SHA-256 of the lines 'element:sorted neighbour ids' (1-based)."""
    h = hashlib.sha256()
    for e, nb in enumerate(neighbours):
        h.update(f"{e + 1}:{','.join(str(x) for x in sorted(nb))}\n".encode())
    return h.hexdigest()


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DSEM_REFERENCE_DIR", "")
    case = os.path.join(ref, "p8-22x22x22")
    with open(os.path.join(case, "DNS-22p8.graph")) as f:
        ne, nm = (int(x) for x in f.readline().split()[:2])
        nbs = [[int(x) for x in f.readline().split()] for _ in range(ne)]
    with open(os.path.join(case, "tgv-22x22x22-p8.mesh")) as f:
        lines = f.read().splitlines()
    nodes = {}
    i = lines.index("nodes") + 1
    while not lines[i].startswith("end"):
        t = lines[i].split()
        nodes[int(t[0])] = [float(x) for x in t[1:4]]
        i += 1
    elems = []
    i = lines.index("elements") + 1
    while not lines[i].startswith("end"):
        elems.append((int(lines[i].split()[0]), [int(x) for x in lines[i + 1].split()]))
        i += 2
    with open(os.path.join(case, "DNS-22p8.graph.part.100")) as f:
        part = [int(x) for x in f.read().split()]
    assert len(part) == ne and 0 <= min(part) and max(part) < 256
    with open(os.path.join(case, "grid_distribution.dat")) as f:
        dist = [(int(t[1]), int(t[2])) for t in (line.split() for line in f) if t]
    assert len(dist) == ne and [r for _, r in dist] == part and max(k for k, _ in dist) < 256
    out = {
        "source": "p8-22x22x22/DNS-22p8.graph, tgv-22x22x22-p8.mesh, DNS-22p8.graph.part.100 and "
                  "grid_distribution.dat of the reference",
        "graph_header": [ne, nm],
        "self_listed": [e + 1 for e in range(ne) if e + 1 in nbs[e]],
        "adjacency_sha256": adjacency_digest(nbs),
        "elements_in_mesh_file": len(elems),
        "corner_sample": {str(eid): [nodes[k] for k in conn] for eid, conn in elems[::SAMPLE]},
        "metis_part_100_b64": base64.b64encode(bytes(part)).decode(),
        "grid_distribution_local_b64": base64.b64encode(bytes(k for k, _ in dist)).decode(),
    }
    with open(os.path.join(HERE, "mesh_22cube_p8.json"), "w") as f:
        json.dump(out, f, indent=0)
    print(f"{len(out['corner_sample'])} sampled elements, {len(out['self_listed'])} self-listed")


if __name__ == "__main__":
    main()
