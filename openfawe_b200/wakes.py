"""Seeded synthetic free wakes for parity tests and benchmarks.

The reference measures on frozen production wakes that it does not ship (``state_<step>.npz``, read by
paper1/scripts/convergence/local_benchmark.py:56-62); these generators stand in for them with the shapes, sizes and
value distributions of the reference's published cases.  Every case returns the arguments of the vortex-batch backend
signature (``points, starts, directions, lengths, gamma, radius, model``) plus the node/edge form.

* ``selftest_sheet``: the wake sheet of the reference's GPU self-test and README speed table
  (apps/studio/openfawe_studio/selftest.py:242-271): 110 nodes per row, 219 segments per row, Lamb-Oseen core 0.075 m,
  circulation linspace(0.5, 1.5), targets on the first 187 rows lifted 0.011 m.
* ``rotor_sheet``: a wing sheet row of 46 nodes (45 spanwise + 46 trailing segments) plus 8 helical rotor rings of 16
  nodes and radius 2 m per shed row (91 + 128 = 219 segments per row), rows convected 0.2 m apart with 0.05 m jitter,
  circulation ~ U(0, 8), Lamb-Oseen core 0.05 m, 20,570 targets on the youngest rows' nodes lifted 0.011 m.
* ``lattice``: 16 spanwise panels x 128 shed rows (4,207 segments), Rosenhead-Moore core 0.05 m, 1,024 targets at the
  three-quarter-chord points of a 1,024-panel wing line over a 26 m span.
* ``ring_wing``: a 64-panel elliptic wing's attached rings with the per-panel column layout of the VSM operators.
* ``wake_batch``: 48 rotor-sheet wakes with log-uniform sizes in [5k, 410k] segments, wind 6-14 m/s setting the row
  spacing, log-uniform target counts in [2,000, 20,570].
"""
import numpy as np

LAMB_OSEEN = 2
ROSENHEAD_MOORE = 5


def _segments(nodes, edges):
    starts = nodes[edges[:, 0]]
    delta = nodes[edges[:, 1]] - starts
    lengths = np.hypot(np.hypot(delta[:, 0], delta[:, 1]), delta[:, 2])
    return starts, delta / lengths[:, None], lengths


def _case(points, nodes, edges, gamma, radius, model, euclid=False, **extra):
    if euclid:      # the self-test's own normalisation: np.linalg.norm, not nested hypot
        starts = nodes[edges[:, 0]]
        vector = nodes[edges[:, 1]] - starts
        lengths = np.linalg.norm(vector, axis=1)
        directions = vector / lengths[:, None]
    else:
        starts, directions, lengths = _segments(nodes, edges)
    return dict(points=np.ascontiguousarray(points, dtype=np.float64), starts=starts, directions=directions,
                lengths=lengths, gamma=np.asarray(gamma, dtype=np.float64), radius=np.asarray(radius, dtype=np.float64),
                model=int(model), nodes=nodes, edges=edges, **extra)


def selftest_sheet(rows, nodes_per_row=110, span=26.0, dx=0.45, seed=0):
    """The reference self-test sheet geometry (selftest.py:242-271), same random stream and formulas."""
    rng = np.random.default_rng(seed)
    y = np.linspace(-span / 2, span / 2, nodes_per_row)
    grid = np.zeros((rows, nodes_per_row, 3))
    for r in range(rows):
        s = r * dx
        grid[r, :, 0] = s + 0.02 * rng.standard_normal(nodes_per_row)
        grid[r, :, 1] = y * (1 + 0.002 * r) + 0.5 * np.sin(0.01 * r)
        grid[r, :, 2] = -0.03 * s + 0.3 * np.sin(y / 3.0 + 0.02 * r)
    nodes = grid.reshape(-1, 3)
    edges = []
    for r in range(rows):
        base = r * nodes_per_row
        k = np.arange(nodes_per_row - 1)
        edges.append(np.column_stack((base + k, base + k + 1)))
        if r + 1 < rows:
            k = np.arange(nodes_per_row)
            edges.append(np.column_stack((base + k, base + nodes_per_row + k)))
    edges = np.concatenate(edges).astype(np.int64)
    targets = grid[:min(rows, 187)].reshape(-1, 3) + np.array([0.0, 0.0, 0.011])
    gamma = np.linspace(0.5, 1.5, len(edges))
    return _case(targets, nodes, edges, gamma, np.full(len(edges), 0.075), LAMB_OSEEN, euclid=True)


ROTOR_HUBS = np.array([[-0.5, y, z] for z in (2.6, -2.6) for y in (-9.75, -3.25, 3.25, 9.75)])


def rotor_sheet(rows, seed=468, targets=20570, wind=10.0, dt=0.02, jitter=0.05, span=26.0, ring_radius=2.0,
                phase_step=0.61, core=0.05):
    """Wing sheet + 8 helical rotor rings per shed row (219 segments per row)."""
    rng = np.random.default_rng(seed)
    spacing = wind * dt
    wing_nodes, ring_nodes, ring_count = 46, 16, len(ROTOR_HUBS)
    per_row = wing_nodes + ring_count * ring_nodes
    y = np.linspace(-span / 2, span / 2, wing_nodes)
    angle0 = 2 * np.pi * np.arange(ring_nodes) / ring_nodes
    nodes = np.zeros((rows, per_row, 3))
    for r in range(rows):
        x = r * spacing
        nodes[r, :wing_nodes, 0] = x
        nodes[r, :wing_nodes, 1] = y
        nodes[r, :wing_nodes, 2] = 0.15 * np.sin(y / 4.0 + 0.05 * r) - 0.01 * x
        angle = angle0 + r * phase_step
        for k, hub in enumerate(ROTOR_HUBS):
            block = nodes[r, wing_nodes + k * ring_nodes: wing_nodes + (k + 1) * ring_nodes]
            block[:, 0] = hub[0] + x
            block[:, 1] = hub[1] + ring_radius * np.cos(angle)
            block[:, 2] = hub[2] + ring_radius * np.sin(angle) - 0.01 * x
    nodes += jitter * rng.standard_normal(nodes.shape)
    flat = nodes.reshape(-1, 3)
    edges = []
    for r in range(rows):
        base = r * per_row
        k = np.arange(wing_nodes - 1)
        edges.append(np.column_stack((base + k, base + k + 1)))
        if r + 1 < rows:
            k = np.arange(wing_nodes)
            edges.append(np.column_stack((base + k, base + per_row + k)))
        for ring in range(ring_count):
            first = base + wing_nodes + ring * ring_nodes
            k = np.arange(ring_nodes)
            edges.append(np.column_stack((first + k, first + (k + 1) % ring_nodes)))
    edges = np.concatenate(edges).astype(np.int64)
    gamma = rng.uniform(0.0, 8.0, len(edges))
    need = min(targets, rows * per_row)
    points = flat[:need] + np.array([0.0, 0.0, 0.011])
    return _case(points, flat, edges, gamma, np.full(len(edges), core), LAMB_OSEEN, rows=rows)


def lattice(seed=1, stations=16, rows=128, targets=1024, span=26.0, wind=10.0, dt=0.02, jitter=0.05, core=0.05):
    """Config-1 lattice: (stations+1) nodes per shed row, spanwise + trailing segments, Rosenhead-Moore core."""
    rng = np.random.default_rng(seed)
    y = np.linspace(-span / 2, span / 2, stations + 1)
    nodes = np.zeros((rows, stations + 1, 3))
    for r in range(rows):
        nodes[r, :, 0] = r * wind * dt
        nodes[r, :, 1] = y
    nodes += jitter * rng.standard_normal(nodes.shape)
    flat = nodes.reshape(-1, 3)
    n = stations + 1
    edges = []
    for r in range(rows):
        k = np.arange(stations)
        edges.append(np.column_stack((r * n + k, r * n + k + 1)))
        if r + 1 < rows:
            k = np.arange(n)
            edges.append(np.column_stack((r * n + k, (r + 1) * n + k)))
    edges = np.concatenate(edges).astype(np.int64)
    gamma = rng.uniform(0.0, 8.0, len(edges))
    panel = np.linspace(-span / 2, span / 2, targets + 1)
    chord = 1.0
    points = np.column_stack((np.full(targets, -chord + 0.75 * chord), 0.5 * (panel[:-1] + panel[1:]),
                              np.full(targets, 0.011)))
    return _case(points, flat, edges, gamma, np.full(len(edges), core), ROSENHEAD_MOORE)


def wake_batch(count=48, seed=48, low=5_000, high=410_000, targets_low=2_000, targets_high=20_570):
    """48 independent rotor-sheet wakes of uneven sizes (wind-speed sweep)."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(low), np.log(high), count))
    winds = rng.uniform(6.0, 14.0, count)
    target_counts = np.exp(rng.uniform(np.log(targets_low), np.log(targets_high), count)).astype(int)
    cases = []
    for k in range(count):
        rows = max(2, int(round(sizes[k] / 219)))
        cases.append(rotor_sheet(rows, seed=seed * 1000 + k, targets=int(target_counts[k]), wind=float(winds[k])))
    return cases


def ring_wing(panels=64, rows=4, span=26.0, chord=2.0, spacing=0.4, seed=64, core=0.05):
    """An elliptic wing's attached vortex rings as the VSM operators use them: (rows+1) x (panels+1) lattice nodes
    (quarter-chord bound line, then rows shed 0.4 m apart), unique undirected segments in first-appearance order, and
    one column per panel listing its rings' segments with the sign of their direction in the ring; edges shared by
    consecutive rings of a panel cancel and are left out (the layout vsm_wake._ring_layout builds,
    src/openfawe/aero/vsm_wake.py:176-221).  Control points at the three-quarter chord lifted 0.01 m."""
    rng = np.random.default_rng(seed)
    y = np.linspace(-span / 2, span / 2, panels + 1)
    c = chord * np.sqrt(np.maximum(1 - (2 * y / span) ** 2, 0.05))
    nodes = np.zeros((rows + 1, panels + 1, 3))
    for r in range(rows + 1):
        nodes[r, :, 0] = 0.25 * c + r * spacing
        nodes[r, :, 1] = y
        nodes[r, :, 2] = 0.02 * r * np.sin(y / 5.0)
    nodes[1:] += 0.01 * rng.standard_normal(nodes[1:].shape)
    flat = nodes.reshape(-1, 3)
    width = panels + 1
    appearance, per_panel = {}, [dict() for _ in range(panels)]
    for i in range(rows):
        for j in range(panels):
            ring = [i * width + j, i * width + j + 1, (i + 1) * width + j + 1, (i + 1) * width + j]
            for a, b in zip(ring, ring[1:] + ring[:1]):
                key = (min(a, b), max(a, b))
                appearance.setdefault(key, len(appearance))
                per_panel[j][key] = per_panel[j].get(key, 0.0) + (1.0 if a < b else -1.0)
    unique, columns = {}, []
    for edges in per_panel:
        column = []
        for key in sorted(edges, key=appearance.__getitem__):
            if edges[key] != 0.0:
                column.append((unique.setdefault(key, len(unique)), edges[key]))
        columns.append(column)
    segments = np.asarray(list(unique), dtype=np.int64).reshape(-1, 2)
    pointer = np.zeros(panels + 1, dtype=np.int64)
    pointer[1:] = np.cumsum([len(col) for col in columns])
    column_segment = np.asarray([k for col in columns for k, _ in col], dtype=np.int64)
    column_sign = np.asarray([v for col in columns for _, v in col], dtype=np.float64)
    yc = 0.5 * (y[:-1] + y[1:])
    cc = chord * np.sqrt(np.maximum(1 - (2 * yc / span) ** 2, 0.05))
    control = np.column_stack((0.75 * cc, yc, np.full(panels, 0.01)))
    case = _case(control, flat, segments, np.ones(len(segments)), np.full(len(segments), core), LAMB_OSEEN)
    case.update(column_ptr=pointer, column_segment=column_segment, column_sign=column_sign)
    return case


def backend_args(case):
    """The positional arguments of the backend signature, without csr and singularity."""
    return (case["points"], case["starts"], case["directions"], case["lengths"], case["gamma"], case["radius"],
            case["model"])
