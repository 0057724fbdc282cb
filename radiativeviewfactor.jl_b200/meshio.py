"""Mesh ingest: Gmsh .msh 4.1 / 2.2 ASCII files -> MeshData (src/MeshIO.jl:94-149).

The reference opens meshes through the Gmsh API (`load_mesh`); Gmsh is not
part of this backend, so this module reads the file format itself.  A 4.1
file carries exactly what the reference asks the API for: the physical
groups and their names ($PhysicalNames, $Entities), the nodes of each entity
($Nodes blocks: a node belongs to the one entity it is classified on, which
is what gmsh.model.mesh.getNodes(dim, tag) returns) and the elements of each
entity by type ($Elements blocks).

What follows the reference step by step:
  * node numbering: every node block in (dim, tag) order, nodes in file order
    (getNodes(), src/MeshIO.jl:208-214);
  * physical groups of dimension surface_dim, named from $PhysicalNames or
    "group_<tag>" (src/MeshIO.jl:216-225); none -> one synthetic group
    "default" over every entity of that dimension, with the next free
    physical tag (src/MeshIO.jl:235-244);
  * per group, per entity of the group, per element type: the supported
    types Line2 (1), Line3 (8), Tri3 (2), Tri6 (9), Quad4 (3), Quad8 (16) and
    Quad9 (10, centre node dropped -> Quad8); an entity in two groups gives
    its elements to both (src/MeshIO.jl:246-310);
  * curve meshes: each line element is flipped (end nodes swapped) when its
    normal at xi = 0 points away from the centroid of the surface next to
    its curve (src/MeshIO.jl:330-600);
  * reverse_normals: the reference's node swaps, including its mid-side
    swaps 5<->7 (Quad8) and 4<->6 (Tri6) (src/MeshIO.jl:613-636);
  * obstruction soups per group (build_group_obs_soups, src/MeshIO.jl:648-685).

Where the reference's order is Julia's Dict / Set iteration order (the groups
of a mesh, src/MeshIO.jl:253; the nodes summed into a surface centroid,
src/MeshIO.jl:388-392), which Julia does not define, this reader takes
ascending tags and ascending node positions: elements come grouped by
ascending physical tag, so the element-level F is a permutation of the
reference's by groups and every group-level result is the same.
.msh 2.2 ASCII files are read too: there an entity is an elementary tag,
its physical groups are those its elements name, and each node is
classified on the lowest-dimensional entity whose elements use it.  Binary
files and other format versions are rejected.
"""
from __future__ import annotations

import math
import os
import shlex
from dataclasses import dataclass, field
from typing import Dict, List, Tuple

import numpy as np

from .mesh import FAMILY_CODES, MeshData, build_group_obs_soups

# Gmsh element type -> (nodes in the file, nodes kept, family); src/MeshIO.jl:26-34
ELEM_INFO = {
    1: (2, 2, "line2"),
    8: (3, 3, "line3"),
    2: (3, 3, "tri3"),
    9: (6, 6, "tri"),
    3: (4, 4, "quad4"),
    16: (8, 8, "quad"),
    10: (9, 8, "quad"),
}
_TYPE_NAMES = {1: "Line2", 8: "Line3", 2: "Tri3", 9: "Tri6", 3: "Quad4", 16: "Quad8", 10: "Quad9"}
# nodes of the other Gmsh element types, to step over their blocks
_OTHER_NODES = {4: 4, 5: 8, 6: 6, 7: 5, 11: 10, 12: 27, 13: 18, 14: 14, 15: 1, 17: 20, 18: 15, 19: 13,
                20: 9, 21: 10, 22: 12, 23: 15, 24: 15, 25: 21, 26: 4, 27: 5, 28: 6, 29: 20, 30: 35, 31: 56}


@dataclass
class MshModel:
    """The parts of a .msh 4.1 file the loader reads."""
    physical_names: Dict[Tuple[int, int], str] = field(default_factory=dict)  # (dim, tag) -> name
    entity_physicals: Dict[Tuple[int, int], List[int]] = field(default_factory=dict)  # (dim, tag) -> tags
    node_blocks: List[Tuple[int, int, np.ndarray, np.ndarray]] = field(default_factory=list)  # dim, tag, tags, xyz
    elem_blocks: List[Tuple[int, int, int, np.ndarray]] = field(default_factory=list)  # dim, tag, type, [tag|nodes]

    def entities(self, dim: int) -> List[int]:
        tags = {t for (d, t) in self.entity_physicals if d == dim}
        tags |= {t for (d, t, *_) in self.node_blocks if d == dim}
        tags |= {t for (d, t, *_) in self.elem_blocks if d == dim}
        return sorted(tags)

    def physical_groups(self, dim: int) -> List[int]:
        tags = {p for (d, _), ps in self.entity_physicals.items() if d == dim for p in ps}
        return sorted(tags)

    def entities_of_group(self, dim: int, ptag: int) -> List[int]:
        return sorted(t for (d, t), ps in self.entity_physicals.items() if d == dim and ptag in ps)

    def max_physical_tag(self) -> int:
        tags = [p for ps in self.entity_physicals.values() for p in ps] + [t for (_, t) in self.physical_names]
        return max(tags, default=0)


def _sections(text: str):
    """Yield (name, lines) for every $Name ... $EndName section."""
    lines = text.splitlines()
    k = 0
    while k < len(lines):
        s = lines[k].strip()
        if s.startswith("$") and not s.startswith("$End"):
            name = s[1:]
            end = "$End" + name
            j = k + 1
            while j < len(lines) and lines[j].strip() != end:
                j += 1
            if j >= len(lines):
                raise ValueError(f"section ${name} has no {end}")
            yield name, lines[k + 1:j]
            k = j + 1
        else:
            k += 1


def read_msh(filename: str) -> MshModel:
    """Parse a Gmsh .msh file, 4.1 or 2.2 ASCII."""
    with open(filename, "rb") as f:
        raw = f.read()
    try:
        text = raw.decode("utf-8")
    except UnicodeDecodeError:
        raise ValueError(f"{filename}: not an ASCII .msh file (binary .msh is not supported)") from None
    sections: Dict[str, List[str]] = {}
    for name, body in _sections(text):
        sections.setdefault(name, body)
    if "MeshFormat" not in sections:
        raise ValueError(f"{filename}: no $MeshFormat section (not a Gmsh .msh file)")
    parts = sections["MeshFormat"][0].split()
    version, ftype = parts[0], int(parts[1])
    if version not in ("4.1", "2.2"):
        raise ValueError(f"{filename}: .msh version {version} is not supported (4.1 or 2.2 ASCII)")
    if ftype != 0:
        raise ValueError(f"{filename}: binary .msh is not supported (4.1 or 2.2 ASCII)")
    model = MshModel()
    body = sections.get("PhysicalNames")
    if body:
        for ln in body[1:1 + int(body[0])]:
            p = shlex.split(ln)
            model.physical_names[(int(p[0]), int(p[1]))] = p[2] if len(p) > 2 else ""
    if version == "4.1":
        if "Entities" in sections:
            _parse_entities(sections["Entities"], model)
        if "Nodes" in sections:
            _parse_nodes(sections["Nodes"], model)
        if "Elements" in sections:
            _parse_elements(sections["Elements"], model)
    elif "Nodes" in sections:
        _parse_v2(sections["Nodes"], sections.get("Elements", ["0"]), model, filename)
    return model


# dimension of each Gmsh element type (points 15; lines 1, 8; surfaces 2, 3,
# 9, 10, 16; the rest are volumes or higher-order types not read here)
_TYPE_DIM = {15: 0, 1: 1, 8: 1, 26: 1, 27: 1, 28: 1, 2: 2, 3: 2, 9: 2, 10: 2, 16: 2, 20: 2, 21: 2, 22: 2, 23: 2,
             24: 2, 25: 2}


def _parse_v2(node_body: List[str], body: List[str], model: MshModel, filename: str):
    """.msh 2.2: elements carry their physical and elementary tags; there are
    no entity blocks, so an entity is an elementary tag of a dimension, it
    belongs to the physical groups its elements name, and a node is
    classified on the lowest-dimensional entity whose elements use it (a
    model point, then a curve, ...), as Gmsh classifies mesh nodes."""
    n_nodes = int(node_body[0].split()[0])
    tags = np.empty(n_nodes, dtype=np.int64)
    xyz = np.empty((n_nodes, 3))
    for a in range(n_nodes):
        v = node_body[1 + a].split()
        tags[a] = int(v[0])
        xyz[a] = [float(v[1]), float(v[2]), float(v[3])]
    n_el = int(body[0].split()[0])
    blocks: Dict[Tuple[int, int, int], list] = {}
    owner: Dict[int, Tuple[int, int]] = {}
    for a in range(n_el):
        v = [int(x) for x in body[1 + a].split()]
        etag, etype, ntags = v[0], v[1], v[2]
        tg = v[3:3 + ntags]
        phys = tg[0] if ntags >= 1 else 0
        ent = tg[1] if ntags >= 2 else 0
        nodes = v[3 + ntags:]
        width = ELEM_INFO[etype][0] if etype in ELEM_INFO else _OTHER_NODES.get(etype, len(nodes))
        if len(nodes) != width:
            raise ValueError(f"{filename}: element {etag} of type {etype} has {len(nodes)} nodes, expected {width}")
        dim = _TYPE_DIM.get(etype, 3)
        ps = model.entity_physicals.setdefault((dim, ent), [])
        if phys and phys not in ps:
            ps.append(phys)
        blocks.setdefault((dim, ent, etype), []).append([etag] + nodes)
        for t in nodes:
            cur = owner.get(t)
            if cur is None or (dim, ent) < cur:
                owner[t] = (dim, ent)
    for (dim, ent, etype), rows in blocks.items():
        model.elem_blocks.append((dim, ent, etype, np.array(rows, dtype=np.int64)))
    per_block: Dict[Tuple[int, int], List[int]] = {}
    for a in range(n_nodes):
        per_block.setdefault(owner.get(int(tags[a]), (3, 0)), []).append(a)
    for (dim, ent), idx in per_block.items():
        model.node_blocks.append((dim, ent, tags[idx], xyz[idx]))


def _parse_entities(body: List[str], model: MshModel):
    counts = [int(x) for x in body[0].split()]
    k = 1
    for dim in range(4):
        for _ in range(counts[dim]):
            v = body[k].split()
            k += 1
            tag = int(v[0])
            at = 4 if dim == 0 else 7  # point: tag x y z; others: tag + bounding box
            n = int(v[at])
            model.entity_physicals[(dim, tag)] = [int(x) for x in v[at + 1:at + 1 + n]]


def _parse_nodes(body: List[str], model: MshModel):
    n_blocks = int(body[0].split()[0])
    k = 1
    for _ in range(n_blocks):
        dim, tag, parametric, n = (int(x) for x in body[k].split())
        k += 1
        tags = np.array([int(body[k + a].split()[0]) for a in range(n)], dtype=np.int64)
        k += n
        xyz = np.array([[float(x) for x in body[k + a].split()[:3]] for a in range(n)],
                       dtype=np.float64).reshape(n, 3)
        k += n
        model.node_blocks.append((dim, tag, tags, xyz))


def _parse_elements(body: List[str], model: MshModel):
    n_blocks = int(body[0].split()[0])
    k = 1
    for _ in range(n_blocks):
        dim, tag, etype, n = (int(x) for x in body[k].split())
        k += 1
        rows = [[int(x) for x in body[k + a].split()] for a in range(n)]
        k += n
        width = ELEM_INFO[etype][0] if etype in ELEM_INFO else _OTHER_NODES.get(etype)
        if width is None:
            width = max((len(r) - 1 for r in rows), default=0)
        if any(len(r) != 1 + width for r in rows):
            raise ValueError(f"element block of type {etype} on entity ({dim}, {tag}): expected {width} nodes "
                             "per element")
        model.elem_blocks.append((dim, tag, etype, np.array(rows, dtype=np.int64).reshape(n, 1 + width)))


def is_xml_vtk(filename: str) -> bool:
    """src/MeshIO.jl:158-170: XML VTK by extension, or a .vtk file whose head
    is XML."""
    ext = os.path.splitext(filename)[1].lower()
    if ext in (".vtu", ".pvtu", ".vts", ".vtr", ".vti", ".vtp"):
        return True
    if ext != ".vtk":
        return False
    with open(filename, "rb") as f:
        head = f.read(512).decode("latin-1")
    return "<?xml" in head or "<VTKFile" in head


def load_vtu(filename: str, surface_dim: int = 2, reverse_normals: bool = False, verbose: bool = True,
             group_field=None) -> MeshData:
    """src/MeshIO.jl:191-206.  The reference reads XML VTK through its ReadVTK
    extension and raises when ReadVTK is not loaded; this backend has no XML
    VTK reader, so it always raises."""
    raise NotImplementedError(
        f"{filename}: reading XML VTK files (.vtu) needs the reference's ReadVTK extension, which this backend "
        "does not provide; write the mesh as Gmsh .msh (4.1 or 2.2 ASCII) and use load_mesh.")


def load_mesh(filename: str, surface_dim: int = 2, reverse_normals: bool = False,
              verbose: bool = True) -> MeshData:
    """src/MeshIO.jl:94-149 for Gmsh .msh 4.1 and 2.2 ASCII files."""
    if not os.path.isfile(filename):
        raise FileNotFoundError(f"Mesh file not found: {filename}")
    if surface_dim not in (1, 2):
        raise ValueError(f"surface_dim must be 1 or 2, got {surface_dim}")
    if is_xml_vtk(filename):  # src/MeshIO.jl:101-103
        return load_vtu(filename, surface_dim, reverse_normals, verbose)
    model = read_msh(filename)
    dim = surface_dim
    # nodes (getNodes(): every entity block, by dimension then tag)
    blocks = sorted(model.node_blocks, key=lambda b: (b[0], b[1]))
    all_tags = np.concatenate([b[2] for b in blocks]) if blocks else np.zeros(0, dtype=np.int64)
    xyz = np.concatenate([b[3] for b in blocks]) if blocks else np.zeros((0, 3))
    tag2pos = {int(t): i + 1 for i, t in enumerate(all_tags)}
    if len(tag2pos) != len(all_tags):
        raise ValueError(f"{filename}: a node tag appears in more than one node block")
    coords = np.asfortranarray(xyz.T)
    # physical groups of the radiating dimension
    names: Dict[int, str] = {}
    for ptag in model.physical_groups(dim):
        nm = model.physical_names.get((dim, ptag), "")
        names[ptag] = nm if nm else f"group_{ptag}"
    group_entities: Dict[int, List[int]] = {p: model.entities_of_group(dim, p) for p in names}
    if not names:  # src/MeshIO.jl:235-244
        ents = model.entities(dim)
        if not ents:
            raise ValueError(f"No entities of dimension {dim} found in mesh; nothing to load.")
        ptag = model.max_physical_tag() + 1
        names = {ptag: "default"}
        group_entities = {ptag: ents}
        if verbose:
            print(f'No physical groups of dimension {dim} found; created a synthetic "default" group over all '
                  f"{len(ents)} entities.")
    by_entity: Dict[int, List[Tuple[int, np.ndarray]]] = {}
    for d, tag, etype, rows in model.elem_blocks:
        if d == dim:
            by_entity.setdefault(tag, []).append((etype, rows))
    elems, fams, groups = [], [], []
    type_counts: Dict[int, int] = {}
    for ptag in sorted(names):
        for ent in group_entities[ptag]:
            for etype, rows in sorted(by_entity.get(ent, []), key=lambda b: b[0]):
                if etype not in ELEM_INFO:
                    continue
                _, keep, fam = ELEM_INFO[etype]
                type_counts[etype] = type_counts.get(etype, 0) + rows.shape[0]
                for r in rows:
                    try:
                        elems.append([tag2pos[int(t)] for t in r[1:1 + keep]])
                    except KeyError as e:
                        raise ValueError(f"{filename}: element {int(r[0])} refers to node {e.args[0]}, "
                                         "which no node block holds") from None
                    fams.append(FAMILY_CODES[fam])
                    groups.append(ptag)
    if not elems:
        present = sorted({t for d, _, t, _ in model.elem_blocks if d == dim})
        supported = "Line2 (1), Line3 (8)" if dim == 1 else "Tri3 (2), Quad4 (3), Tri6 (9), Quad8 (16), Quad9 (10)"
        raise ValueError(f"No supported elements found in physical groups (dimension {dim}).\n"
                         f"Supported types (1st or 2nd order): {supported}\n"
                         f"Element types present at dimension {dim}: {present}")
    en = np.zeros((len(elems), 8), dtype=np.int32)
    for e, el in enumerate(elems):
        en[e, :len(el)] = el
    md = MeshData(coords, en, np.asarray(fams, dtype=np.int8), np.asarray(groups, dtype=np.int32), names, {}, dim)
    if dim == 1:
        n_flip = orient_line_normals(md, model, tag2pos, group_entities)
        if verbose and n_flip:
            print(f"  Reoriented {n_flip} Line3 element(s) to point toward transfinite surface interior.")
    if reverse_normals:
        reverse_all_normals(md)
        if verbose:
            print("  All normals reversed.")
    md.group_tri_soup = {int(k): np.ascontiguousarray(v) for k, v in build_group_obs_soups(md).items()}
    if verbose:
        c = {f: int((md.elem_family == FAMILY_CODES[f]).sum()) for f in FAMILY_CODES}
        if dim == 2:
            print(f"Loaded {md.n_elems} surface elements (quad8: {c['quad']}, quad4: {c['quad4']}, "
                  f"tri6: {c['tri']}, tri3: {c['tri3']}) in {len(names)} physical group(s).")
        else:
            print(f"Loaded {md.n_elems} curve elements (line3: {c['line3']}, line2: {c['line2']}) "
                  f"in {len(names)} physical group(s).")
        for t in sorted(type_counts):
            print(f"  Element type {_TYPE_NAMES[t]}: {type_counts[t]} elements")
    return md


def _centroid(coords: np.ndarray, positions) -> np.ndarray:
    p = np.asarray(sorted(positions), dtype=np.int64) - 1
    return np.array([sum(coords[c, p]) / len(p) for c in range(3)])


def orient_line_normals(md: MeshData, model: MshModel, tag2pos: Dict[int, int],
                        group_entities: Dict[int, List[int]]) -> int:
    """src/MeshIO.jl:469-600 (with _build_curve_to_surface_centroid, :330-450):
    flips line elements whose normal at xi = 0, n = (-dy, dx) / |t| with t
    from node 1 to node 2, points away from the centroid of the surface next
    to the element's curve.  Returns the number of flipped elements."""
    coords = md.coords
    line_fams = (FAMILY_CODES["line2"], FAMILY_CODES["line3"])
    curve_ents = set()
    for ptag, ents in group_entities.items():
        first = np.flatnonzero(md.elem_group == ptag)
        if first.size and int(md.elem_family[first[0]]) in line_fams:
            curve_ents.update(ents)
    # nodes classified on each curve (getNodes(1, ent): interior nodes only)
    curve_nodes: Dict[int, set] = {}
    for d, tag, tags, _ in model.node_blocks:
        if d == 1 and tag in curve_ents:
            curve_nodes.setdefault(tag, set()).update(tag2pos[int(t)] for t in tags)
    pos_to_curve: Dict[int, int] = {}
    for ent in sorted(curve_nodes):
        for p in curve_nodes[ent]:
            pos_to_curve.setdefault(p, ent)
    # surfaces: those of physical groups of dimension 2, else every surface
    surf_ents = sorted({e for p in model.physical_groups(2) for e in model.entities_of_group(2, p)})
    if not surf_ents:
        surf_ents = model.entities(2)
    surf_nodes: Dict[int, set] = {}
    for d, tag, etype, rows in model.elem_blocks:
        if d == 2 and tag in surf_ents:
            s = surf_nodes.setdefault(tag, set())
            for t in rows[:, 1:].ravel():
                p = tag2pos.get(int(t))
                if p is not None:
                    s.add(p)
    surf_centroid = {s: _centroid(coords, ns) for s, ns in surf_nodes.items() if ns}
    curve_to_surf: Dict[int, np.ndarray] = {}
    for ent, cn in curve_nodes.items():
        if not cn:
            continue
        cc = _centroid(coords, cn)
        best, best_d = None, math.inf
        for s in sorted(surf_centroid):
            if cn & surf_nodes[s]:
                dd = float(np.sum((cc - surf_centroid[s]) ** 2))
                if dd < best_d:
                    best, best_d = s, dd
        if best is not None:
            curve_to_surf[ent] = surf_centroid[best]
    n_flip = 0
    en = md.elem_nodes
    for e in range(md.n_elems):
        f = int(md.elem_family[e])
        if f not in line_fams:
            continue
        ent = pos_to_curve.get(int(en[e, 0]), 0) or pos_to_curve.get(int(en[e, 1]), 0)
        if not ent or ent not in curve_to_surf:
            continue
        a, b = int(en[e, 0]) - 1, int(en[e, 1]) - 1
        if f == FAMILY_CODES["line3"]:
            mid = coords[:, int(en[e, 2]) - 1]
        else:
            mid = np.array([0.5 * (coords[c, a] + coords[c, b]) for c in range(3)])
        dx = coords[0, b] - coords[0, a]
        dy = coords[1, b] - coords[1, a]
        tlen = math.sqrt(dx * dx + dy * dy)
        if tlen < np.finfo(np.float64).eps:
            continue
        n = np.array([-dy / tlen, dx / tlen, 0.0])
        if float(np.dot(n, curve_to_surf[ent] - mid)) < 0.0:
            en[e, 0], en[e, 1] = en[e, 1], en[e, 0]
            n_flip += 1
    return n_flip


def reverse_all_normals(md: MeshData):
    """src/MeshIO.jl:613-636, node swaps as the reference makes them."""
    en = md.elem_nodes
    for e in range(md.n_elems):
        f = int(md.elem_family[e])
        sw = {FAMILY_CODES["line2"]: [(0, 1)], FAMILY_CODES["line3"]: [(0, 1)],
              FAMILY_CODES["quad"]: [(0, 2), (4, 6)], FAMILY_CODES["quad4"]: [(0, 2)],
              FAMILY_CODES["tri"]: [(0, 2), (3, 5)], FAMILY_CODES["tri3"]: [(0, 2)]}[f]
        for a, b in sw:
            en[e, a], en[e, b] = en[e, b], en[e, a]


def write_msh(filename: str, md: MeshData, extra_surfaces=None):
    """Write a MeshData as a .msh 4.1 ASCII file: one entity per group (of the
    mesh's dimension, physical tag = group tag, named), every node classified
    on the entity of the first element that uses it.  extra_surfaces: list of
    (node positions (1-based), elements as (gmsh type, node positions)) put on
    additional unnamed surface entities without a physical group."""
    dim = md.mesh_dim
    gtype = {FAMILY_CODES["quad"]: 16, FAMILY_CODES["quad4"]: 3, FAMILY_CODES["tri"]: 9,
             FAMILY_CODES["tri3"]: 2, FAMILY_CODES["line3"]: 8, FAMILY_CODES["line2"]: 1}
    nkeep = {16: 8, 3: 4, 9: 6, 2: 3, 8: 3, 1: 2, 10: 9}
    tags = sorted(md.group_tags)
    ent_of = {g: k + 1 for k, g in enumerate(tags)}
    owner = {}
    for e in range(md.n_elems):
        t = gtype[int(md.elem_family[e])]
        for p in md.elem_nodes[e, :nkeep[t]]:
            owner.setdefault(int(p), (dim, ent_of[int(md.elem_group[e])]))
    extra = list(extra_surfaces or [])
    for k, (_, els) in enumerate(extra):
        for t, nodes in els:
            for p in nodes:
                owner.setdefault(int(p), (2, len(tags) + k + 1))
    Nn = md.coords.shape[1]
    for p in range(1, Nn + 1):
        owner.setdefault(p, (dim, 1))
    out = ["$MeshFormat", "4.1 0 8", "$EndMeshFormat", "$PhysicalNames", str(len(tags))]
    out += [f'{dim} {g} "{md.group_tags[g]}"' for g in tags]
    out.append("$EndPhysicalNames")
    n_ent = [0, 0, 0, 0]
    n_ent[dim] += len(tags)
    n_ent[2] += len(extra)
    out += ["$Entities", " ".join(map(str, n_ent))]
    lo, hi = md.coords.min(axis=1), md.coords.max(axis=1)
    box = " ".join(repr(float(x)) for x in (*lo, *hi))
    ents = [(dim, ent_of[g], [g]) for g in tags] + [(2, len(tags) + k + 1, []) for k in range(len(extra))]
    for d in (1, 2):
        for dd, tag, phys in ents:
            if dd == d:
                out.append(f"{tag} {box} {len(phys)} {' '.join(map(str, phys))} 0".replace("  ", " "))
    out.append("$EndEntities")
    blocks: Dict[Tuple[int, int], List[int]] = {}
    for p in range(1, Nn + 1):
        blocks.setdefault(owner[p], []).append(p)
    out += ["$Nodes", f"{len(blocks)} {Nn} 1 {Nn}"]
    for (d, tag) in sorted(blocks):
        ps = blocks[(d, tag)]
        out.append(f"{d} {tag} 0 {len(ps)}")
        out += [str(p) for p in ps]
        out += [" ".join(repr(float(md.coords[c, p - 1])) for c in range(3)) for p in ps]
    out.append("$EndNodes")
    eblocks: Dict[Tuple[int, int, int], List[List[int]]] = {}
    for e in range(md.n_elems):
        t = gtype[int(md.elem_family[e])]
        eblocks.setdefault((dim, ent_of[int(md.elem_group[e])], t), []).append(
            [int(x) for x in md.elem_nodes[e, :nkeep[t]]])
    for k, (_, els) in enumerate(extra):
        for t, nodes in els:
            eblocks.setdefault((2, len(tags) + k + 1, t), []).append([int(x) for x in nodes])
    n_el = sum(len(v) for v in eblocks.values())
    out += ["$Elements", f"{len(eblocks)} {n_el} 1 {n_el}"]
    tag = 1
    for (d, ent, t), rows in eblocks.items():
        out.append(f"{d} {ent} {t} {len(rows)}")
        for r in rows:
            out.append(f"{tag} " + " ".join(map(str, r)))
            tag += 1
    out.append("$EndElements")
    with open(filename, "w") as f:
        f.write("\n".join(out) + "\n")
