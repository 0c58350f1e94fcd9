"""Parametric panel meshes and HAMS input decks for the benchmark cases.

Meshes follow HAMS-MREL's conventions (src/ReadPanelMesh.f90,
src/NormalProcess.f90): quadrilateral panels with 1-based node ids, normals
from the diagonal cross product (P4-P2) x (P3-P1) pointing into the body, and
the innermost bottom ring written as quads with a repeated centre node
(degenerate edges are skipped by the panel integrals, SingularIntgr.f90:416).

Cases (all seeded, no external data):
  c1  truncated cylinder R=5, T=10, 40 x 15 side + 40 x 5 bottom = 800 panels, infinite depth
  c2  3 x 3 array of cylinders R=4, T=8 at 20 m, 40 x 10 + 40 x 5 = 600 panels each (5,400), h = 50 m
  c3  128 single/two-body cases (cylinders or boxes, 200-3000 panels, half with a water-plane lid)
  c5  6 x 6 array of cylinders R=3, T=6 at 12 m, 40 x 9 + 40 x 5 = 560 panels each (20,160), h = 40 m
"""
import os

import numpy as np


def _orient(nodes, quad, outward):
    """Order a quad so that (P4-P2) x (P3-P1) points against `outward` (into the body)."""
    p = nodes[np.array(quad) - 1]
    un = np.cross(p[3] - p[1], p[2] - p[0])
    if np.dot(un, outward) > 0:
        quad = [quad[0], quad[3], quad[2], quad[1]]
    return quad


def cylinder(radius, draft, n_theta, n_z, n_r, x0=0.0, y0=0.0):
    """Truncated vertical cylinder: side n_theta x n_z quads, flat bottom n_theta x n_r quads.

    Returns (xyz (ntnd,3), ncn (n,), ncon (n,4)) with 1-based node ids.
    """
    th = 2.0 * np.pi * np.arange(n_theta) / n_theta
    nodes = []
    for k in range(n_z + 1):  # side rings from z = 0 down to z = -draft
        z = -draft * k / n_z
        for t in th:
            nodes.append((x0 + radius * np.cos(t), y0 + radius * np.sin(t), z))
    ring_id = lambda k, i: k * n_theta + (i % n_theta) + 1
    bottom = [ring_id(n_z, i) for i in range(n_theta)]  # r = R ring at z = -draft
    rings = [bottom]
    for m in range(1, n_r):  # inner rings
        r = radius * (n_r - m) / n_r
        ids = []
        for t in th:
            nodes.append((x0 + r * np.cos(t), y0 + r * np.sin(t), -draft))
            ids.append(len(nodes))
        rings.append(ids)
    nodes.append((x0, y0, -draft))
    centre = len(nodes)
    nodes = np.array(nodes, dtype=np.float64)
    quads = []
    for k in range(n_z):
        for i in range(n_theta):
            q = [ring_id(k, i), ring_id(k, i + 1), ring_id(k + 1, i + 1), ring_id(k + 1, i)]
            tc = th[i] + np.pi / n_theta
            quads.append(_orient(nodes, q, np.array([np.cos(tc), np.sin(tc), 0.0])))
    down = np.array([0.0, 0.0, -1.0])
    for m in range(n_r):
        outer = rings[m]
        for i in range(n_theta):
            a, b = outer[i], outer[(i + 1) % n_theta]
            if m < n_r - 1:
                inner = rings[m + 1]
                q = [a, b, inner[(i + 1) % n_theta], inner[i]]
            else:
                q = [a, b, centre, centre]
            quads.append(_orient(nodes, q, down))
    ncon = np.array(quads, dtype=np.int32)
    return nodes, np.full(len(quads), 4, dtype=np.int32), ncon


def box(length, beam, draft, n_l, n_b, n_z, x0=0.0, y0=0.0):
    """Rectangular barge: four sides and a bottom, all quads, normals into the body."""
    xs = np.linspace(-length / 2, length / 2, n_l + 1) + x0
    ys = np.linspace(-beam / 2, beam / 2, n_b + 1) + y0
    zs = np.linspace(0.0, -draft, n_z + 1)
    nodes, index = [], {}

    def nid(p):
        key = tuple(np.round(p, 12))
        if key not in index:
            nodes.append(p)
            index[key] = len(nodes)
        return index[key]

    quads, outs = [], []
    for k in range(n_z):
        for i in range(n_l):  # y = -B/2 and y = +B/2 faces
            for yv, s in ((ys[0], -1.0), (ys[-1], 1.0)):
                q = [nid((xs[i], yv, zs[k])), nid((xs[i + 1], yv, zs[k])), nid((xs[i + 1], yv, zs[k + 1])),
                     nid((xs[i], yv, zs[k + 1]))]
                quads.append(q)
                outs.append((0.0, s, 0.0))
        for j in range(n_b):  # x = -L/2 and x = +L/2 faces
            for xv, s in ((xs[0], -1.0), (xs[-1], 1.0)):
                q = [nid((xv, ys[j], zs[k])), nid((xv, ys[j + 1], zs[k])), nid((xv, ys[j + 1], zs[k + 1])),
                     nid((xv, ys[j], zs[k + 1]))]
                quads.append(q)
                outs.append((s, 0.0, 0.0))
    for i in range(n_l):
        for j in range(n_b):
            q = [nid((xs[i], ys[j], -draft)), nid((xs[i + 1], ys[j], -draft)), nid((xs[i + 1], ys[j + 1], -draft)),
                 nid((xs[i], ys[j + 1], -draft))]
            quads.append(q)
            outs.append((0.0, 0.0, -1.0))
    nodes = np.array(nodes, dtype=np.float64)
    quads = [_orient(nodes, q, np.array(o)) for q, o in zip(quads, outs)]
    return nodes, np.full(len(quads), 4, dtype=np.int32), np.array(quads, dtype=np.int32)


def disc_lid(radius, n_theta, n_r, x0=0.0, y0=0.0):
    """Interior water-plane lid (z = 0) of a cylinder; normals point down like the bottom."""
    nodes, ncn, ncon = cylinder(radius, 1.0, n_theta, 1, n_r, x0, y0)
    # keep only the bottom rings, lifted to z = 0
    keep = ncon[n_theta:]
    used = np.unique(keep)
    remap = np.zeros(nodes.shape[0] + 1, dtype=np.int32)
    remap[used] = np.arange(1, used.size + 1)
    lid_nodes = nodes[used - 1].copy()
    lid_nodes[:, 2] = 0.0
    return lid_nodes, np.full(keep.shape[0], 4, dtype=np.int32), remap[keep]


def rect_lid(length, beam, n_l, n_b, x0=0.0, y0=0.0):
    xs = np.linspace(-length / 2, length / 2, n_l + 1) + x0
    ys = np.linspace(-beam / 2, beam / 2, n_b + 1) + y0
    nodes = np.array([(x, y, 0.0) for y in ys for x in xs])
    nid = lambda i, j: j * (n_l + 1) + i + 1
    quads = []
    for i in range(n_l):
        for j in range(n_b):
            quads.append(_orient(nodes, [nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)],
                                 np.array([0.0, 0.0, -1.0])))
    return nodes, np.full(len(quads), 4, dtype=np.int32), np.array(quads, dtype=np.int32)


def combine(bodies):
    """Stack body meshes into the combined arrays (BuildCombinedArrays order)."""
    xyz, ncn, ncon, counts = [], [], [], []
    off = 0
    for nodes, nc, con in bodies:
        xyz.append(nodes)
        ncn.append(nc)
        ncon.append(con + off)
        counts.append(nc.size)
        off += nodes.shape[0]
    return np.vstack(xyz), np.concatenate(ncn), np.vstack(ncon), np.array(counts, dtype=np.int32)


def case_c1():
    """One cylinder R=5, T=10, 800 panels, infinite depth."""
    return dict(name="c1", bodies=[cylinder(5.0, 10.0, 40, 15, 5)], centres=[(0.0, 0.0, 0.0)], depth=-1.0,
                omegas=np.linspace(0.1, 3.0, 30), betas_deg=[0.0])


def case_c2():
    """3 x 3 cylinders R=4, T=8 at 20 m, 600 panels each (5,400), h = 50 m."""
    bodies, centres = [], []
    for iy in range(3):
        for ix in range(3):
            x0, y0 = 20.0 * ix, 20.0 * iy
            bodies.append(cylinder(4.0, 8.0, 40, 10, 5, x0, y0))
            centres.append((x0, y0, 0.0))
    return dict(name="c2", bodies=bodies, centres=centres, depth=50.0, omegas=np.linspace(0.2, 2.5, 40),
                betas_deg=[0.0, 30.0, 60.0, 90.0])


def case_c5():
    """6 x 6 cylinders R=3, T=6 at 12 m, 560 panels each (20,160), h = 40 m."""
    bodies, centres = [], []
    for iy in range(6):
        for ix in range(6):
            x0, y0 = 12.0 * ix, 12.0 * iy
            bodies.append(cylinder(3.0, 6.0, 40, 9, 5, x0, y0))
            centres.append((x0, y0, 0.0))
    return dict(name="c5", bodies=bodies, centres=centres, depth=40.0, omegas=np.linspace(0.2, 2.5, 24),
                betas_deg=[0.0, 45.0, 90.0])


def case_c3(seed):
    """Heterogeneous case `seed` of 128: one or two random bodies, half of the cases with lids."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nbody = 1 if rng.random() < 0.5 else 2
    lid = rng.random() < 0.5
    depth = -1.0 if rng.random() < 0.5 else float(rng.uniform(30.0, 200.0))
    bodies, lids, centres = [], [], []
    for b in range(nbody):
        target = int(rng.integers(200, 3001))
        x0 = 0.0 if b == 0 else float(rng.uniform(40.0, 80.0))
        if rng.random() < 0.5:
            r, t = float(rng.uniform(2, 8)), float(rng.uniform(3, 12))
            nt = max(8, int(round(np.sqrt(target / 2.0) * 2 / 4)) * 4)
            nz = max(2, target // (2 * nt))
            nr = max(2, (target - nt * nz) // nt)
            bodies.append(cylinder(r, t, nt, nz, nr, x0, 0.0))
            if lid:
                lids.append(disc_lid(r, nt, max(1, nr // 2), x0, 0.0))
        else:
            L, B, T = float(rng.uniform(10, 40)), float(rng.uniform(5, 15)), float(rng.uniform(2, 8))
            s = np.sqrt(target / (2 * (L + B) * T + L * B))
            nl, nb, nz = max(2, int(L * s)), max(2, int(B * s)), max(2, int(T * s))
            bodies.append(box(L, B, T, nl, nb, nz, x0, 0.0))
            if lid:
                lids.append(rect_lid(L * 0.98, B * 0.98, max(1, nl // 2), max(1, nb // 2), x0, 0.0))
        centres.append((x0, 0.0, 0.0))
    return dict(name=f"c3_{seed}", bodies=bodies, lids=lids if lid else None, centres=centres, depth=depth,
                omegas=np.linspace(0.1, 3.0, 16), betas_deg=[0.0])


def write_pnl(path, nodes, ncn, ncon, title="Hull Mesh", isx=0, isy=0):
    """.pnl file in the layout ReadBodyMesh reads (ReadPanelMesh.f90:46-99); isx / isy = 1 marks a
    half mesh (the part x >= 0 or y >= 0 of a body symmetric in that plane)."""
    with open(path, "w") as f:
        f.write(f"    --------------{title} File---------------\n \n")
        f.write("    # Number of Panels, Nodes, X-Symmetry and Y-Symmetry\n")
        f.write(f"{ncn.size:12d}{nodes.shape[0]:12d}{isx:12d}{isy:12d}\n \n")
        f.write("    # Start Definition of Node Coordinates     ! node_number   x   y   z\n")
        for i, (x, y, z) in enumerate(nodes):
            f.write(f"{i + 1:5d}{x:18.6f}{y:18.6f}{z:18.6f}\n")
        f.write("    # End Definition of Node Coordinates\n \n")
        f.write("  # Start Definition of Node Relations   ! panel_number  number_of_vertices   Vertex1_ID ...\n")
        for i in range(ncn.size):
            f.write(f"{i + 1:5d}{ncn[i]:9d}" + "".join(f"{v:14d}" for v in ncon[i, :ncn[i]]) + "\n")
        f.write("    # End Definition of Node Relations\n \n    --------------End Hull Mesh File---------------\n")


def write_deck(directory, case, nthread=8):
    """ControlFile.in, HullMesh[_k].pnl and Hydrostatic[_k].in for `case` (input frequency type 3;
    case["isx"] / case["isy"] = 1 for half meshes)."""
    os.makedirs(directory, exist_ok=True)
    nb = len(case["bodies"])
    multi = nb > 1
    lids = case.get("lids")
    for b, (nodes, ncn, ncon) in enumerate(case["bodies"]):
        # bodies are written in global coordinates with LCS = 0
        write_pnl(os.path.join(directory, f"HullMesh_{b + 1}.pnl" if multi else "HullMesh.pnl"), nodes, ncn, ncon,
                  isx=case.get("isx", 0), isy=case.get("isy", 0))
        with open(os.path.join(directory, f"Hydrostatic_{b + 1}.in" if multi else "Hydrostatic.in"), "w") as f:
            f.write(" Center of Gravity:\n  0.0  0.0  0.0\n")
            for title in ("Body Mass Matrix:", "External Linear Damping Matrix:", "External Quadratic Damping Matrix:",
                          "Hydrostatic Restoring Matrix:", "External Restoring Matrix:"):
                f.write(f" {title}\n" + "".join("  0.00000E+00" * 6 + "\n" for _ in range(6)))
        if lids:
            lnodes, lncn, lncon = lids[b]
            write_pnl(os.path.join(directory, f"WaterPlaneMesh_{b + 1}.pnl" if multi else "WaterPlaneMesh.pnl"),
                      lnodes, lncn, lncon, title="WaterPlane Mesh", isx=case.get("isx", 0), isy=case.get("isy", 0))
    om = case["omegas"]
    with open(os.path.join(directory, "ControlFile.in"), "w") as f:
        f.write("   --------------HAMS Control file---------------\n\n")
        f.write(f"   Waterdepth  {case['depth']:.6f}D0\n\n")
        f.write("   #Start Definition of Wave Frequencies\n")
        f.write("    0_inf_frequency_limits      0\n")
        f.write("    Input_frequency_type        3\n")
        f.write("    Output_frequency_type       3\n")
        f.write(f"    Number_of_frequencies      {len(om)}\n")
        f.write("    " + " ".join(f"{w:.10f}" for w in om) + "\n")
        f.write("   #End Definition of Wave Frequencies\n\n")
        if multi:
            f.write("   # Start of definition of bodies for multi-body interaction\n")
            f.write(f"    Number_of_bodies          {nb}\n")
            for b in range(nb):
                f.write(f"    {'LCS_' + str(b + 1):<22s}" + "".join(f"{0.0:12.3f}" for _ in range(4)) + "\n")
            f.write("   # End of definition of bodies for multi-body interaction\n\n")
        else:
            f.write("   #Start Definition of Wave Headings\n")
        if multi:
            f.write("   #Start Definition of Wave Headings\n")
        f.write(f"    Number_of_headings        {len(case['betas_deg'])}\n")
        f.write("    " + " ".join(f"{b:.6f}" for b in case["betas_deg"]) + "\n")
        f.write("   #End Definition of Wave Headings\n\n")
        for b, c in enumerate(case["centres"]):
            label = f"Reference_body_center_{b + 1}" if multi else "Reference_body_center"
            f.write(f"    {label:<24s}" + "".join(f"{v:12.3f}" for v in c) + "\n")
        f.write("    Reference_body_length   1.0D0\n")
        f.write("    Wave_diffrac_solution    1\n")
        f.write(f"    If_remove_irr_freq       {1 if lids else 0}\n")
        f.write(f"    Number of threads       {nthread}\n\n")
        f.write("   #Start Definition of Pressure and/or Elevation (PE)\n")
        f.write("    Number_of_field_points     0\n")
        f.write("   #End Definition of Pressure and/or Elevation\n\n")
        f.write("   ----------End HAMS Control file---------------\n")
