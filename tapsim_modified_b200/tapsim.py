"""Host-side mirror of the reference's hot-path interface over the C ABI.

Grid collects what Process::evaporation (tapsim/process.cpp:441-1124) calls
on Grid_3d::Table, Surface_3d::Table and Trajectory_3d, backed by one device
handle.  EvaporationOptions reads tapsim.ini with the reference's keys and
strictness (Process::EvaporationOptions::setDefaults, process.cpp:206-439),
and Evaporation runs the event loop with its voltage queue and results log.
"""
from __future__ import annotations

import ctypes as C
import math
import struct
from collections import deque
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _native as N

E_CHARGE = 1.60217733e-19   # Trajectory_3d::eCharge (trajectory_3d.h:91)
AMU2KG = 1.660538782e-27     # Trajectory_3d::amu2kg (trajectory_3d.h:93)


class Mesh:
    """Host mesh (tg_mesh): node set, Delaunay tetrahedra, FP64 Voronoi couplings."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        self._desc = N.tg_mesh_desc()
        nnz = C.c_int32()
        N.check(N.lib().tg_mesh_describe(self._h, C.byref(self._desc), C.byref(nnz)))
        self.nnz = nnz.value

    @staticmethod
    def tip_params(**kw) -> N.tg_tip_params:
        p = N.tg_tip_params()
        N.lib().tg_tip_params_default(C.byref(p))
        for k, v in kw.items():
            if not hasattr(p, k):
                raise KeyError(k)
            setattr(p, k, v)
        return p

    @classmethod
    def from_tip(cls, threads: int = 0, **kw) -> "Mesh":
        h = C.c_void_p()
        N.check(N.lib().tg_mesh_from_tip(C.byref(cls.tip_params(**kw)), threads, C.byref(h)))
        return cls(h)

    @classmethod
    def from_files(cls, node_file: str, config_file: str, threads: int = 0) -> "Mesh":
        h = C.c_void_p()
        N.check(N.lib().tg_mesh_from_files(str(node_file).encode(), str(config_file).encode(), threads, C.byref(h)))
        return cls(h)

    @staticmethod
    def sample_params(**kw) -> N.tg_sample_params:
        p = N.tg_sample_params()
        N.lib().tg_sample_params_default(C.byref(p))
        for k, v in kw.items():
            if not hasattr(p, k):
                raise KeyError(k)
            setattr(p, k, v)
        return p

    @classmethod
    def from_sample(cls, sample_file: str, config_file: str | None = None, threads: int = 0, **kw) -> "Mesh":
        """MeshGen's role (meshgen/meshgen.cpp:2506-3986): graded vacuum and
        the box's marked boundary nodes around the sample in a node file, the
        sample appended last, then the Delaunay mesh and couplings.  Without
        config_file the mesh takes meshgen's configuration template
        (tg_mesh_from_sample)."""
        h = C.c_void_p()
        cfg = str(config_file).encode() if config_file else None
        N.check(N.lib().tg_mesh_from_sample(str(sample_file).encode(), cfg, C.byref(cls.sample_params(**kw)), threads,
                                            C.byref(h)))
        return cls(h)

    @classmethod
    def from_dump(cls, dump_file: str, config_file: str | None = None) -> "Mesh":
        h = C.c_void_p()
        cfg = str(config_file).encode() if config_file else None
        N.check(N.lib().tg_mesh_from_dump(str(dump_file).encode(), cfg, C.byref(h)))
        return cls(h)

    def close(self):
        if self._h:
            N.lib().tg_mesh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def desc(self) -> N.tg_mesh_desc:
        return self._desc

    @property
    def num_nodes(self) -> int:
        return self._desc.num_nodes

    @property
    def temperature(self) -> float:
        """TEMPERATURE of the mesh's configuration [K]."""
        return float(N.lib().tg_mesh_temperature(self._h))

    def arrays(self) -> dict:
        """Copies of the description arrays (node-file order)."""
        d = self._desc
        n, nnz, nt = d.num_nodes, self.nnz, d.num_tets

        def arr(p, dtype, count):
            if not p:
                return None
            ct = np.ctypeslib.as_ctypes_type(np.dtype(dtype))
            return np.ctypeslib.as_array((ct * count).from_address(p)).copy()

        types = [d.types[k] for k in range(d.num_types)]
        return {
            "xyz": arr(d.xyz, np.float32, 3 * n).reshape(n, 3),
            "type": arr(d.type_id, np.int8, n),
            "hull": arr(d.hull, np.uint8, n),
            "phi": arr(d.phi, np.float32, n),
            "row_ptr": arr(d.row_ptr, np.int32, n + 1),
            "col": arr(d.col, np.int32, nnz),
            "coupling": arr(d.coupling, np.float64, nnz),
            "geom": arr(d.geom, np.float64, nnz),
            "area_pos": arr(d.area_pos, np.uint8, nnz),
            "volume": arr(d.volume, np.float64, n),
            "tet_v": arr(d.tet_v, np.int32, 4 * nt).reshape(nt, 4) if nt else None,
            "tet_n": arr(d.tet_n, np.int32, 4 * nt).reshape(nt, 4) if nt else None,
            "node_tet": arr(d.node_tet, np.int32, n),
            "types": {t.id: {f: getattr(t, f) for f, _ in N.tg_type._fields_} for t in types},
        }

    def numbers(self) -> np.ndarray:
        """Grid_3d::Node::number of every node (the node file's or dump's
        unique numbers; index + 1 for a generated tip)."""
        out = np.empty(self._desc.num_nodes, np.uint32)
        N.check(N.lib().tg_mesh_numbers(self._h, N.ptr(out)))
        return out

    def write_node_file(self, path: str, binary: bool = True):
        N.check(N.lib().tg_mesh_write_node_file(self._h, str(path).encode(), int(binary)))

    @property
    def dump_index(self) -> int:
        """LAST_INDEX of the dump the mesh was read from (0 otherwise)."""
        return int(N.lib().tg_mesh_dump_index(self._h))

    def write_grid_nodes(self, path: str, phi: np.ndarray | None = None, binary: bool = False):
        """File_Io::writeGeomGrid (file_io.cpp:765-820): the node file with
        numbers and potentials (phi: float potentials, None: the mesh's own),
        as a relaxation writes it (ASCII by default, tapsim.cpp:129-139)."""
        p = None if phi is None else np.ascontiguousarray(phi, np.float32)
        N.check(N.lib().tg_mesh_write_grid_nodes(self._h, str(path).encode(), int(binary), N.ptr(p)))

    def write_config(self, path: str):
        N.check(N.lib().tg_mesh_write_config(self._h, str(path).encode()))

    def write_dump(self, path: str, phi: np.ndarray | None = None):
        p = None if phi is None else np.ascontiguousarray(phi, np.float32)
        N.check(N.lib().tg_mesh_write_dump(self._h, str(path).encode(), N.ptr(p)))


def path_length(impact: N.tg_impact, cap: int) -> int:
    """Points a flight's path holds: start, accepted steps, extrapolated
    point; none when the start is outside the mesh; at most cap kept."""
    return 0 if impact.status == -1 else min(impact.steps + 2, cap)


def trace_opts(time_step=1e-14, min_time_step=1e-16, error_threshold=1e-6, max_steps=100000, stepper_limit=200,
               walk_limit=100000, integrator=1, stepper=1, precision=0, fp64_radius=0.0) -> N.tg_trace_opts:
    """Trajectory options; integrator / stepper are TRAJECTORY_INTEGRATOR_TYPE
    (0 Euler, 1 Cash-Karp) and TRAJECTORY_STEPPER_TYPE (0 none, 1 error-
    restricted, 2 geometry-restricted, 3 adaptive); precision 0 FP64, 1 FP32,
    2 FP64 within fp64_radius [m] of the start and FP32 beyond."""
    return N.tg_trace_opts(time_step, min_time_step, error_threshold, max_steps, stepper_limit, walk_limit,
                           integrator, stepper, precision, fp64_radius)


def solve_opts(rel_tol=1e-8, max_outer=20, max_inner=4000, inner_rtol=1e-4, warm_start=0,
               preconditioner=0, inner_precision=0) -> N.tg_solve_opts:
    """preconditioner: 0 Jacobi, 1 multigrid; inner_precision: 0 FP32, 1 FP64
    inner iterations (tg_solve_opts)."""
    return N.tg_solve_opts(rel_tol, max_outer, max_inner, inner_rtol, warm_start, preconditioner, inner_precision)


class Grid:
    """Device state of one mesh: Grid_3d::Table + Surface_3d::Table + flights."""

    def __init__(self, mesh: Mesh):
        self.mesh = mesh
        self._h = C.c_void_p()
        N.check(N.lib().tg_create(C.byref(mesh.desc), C.byref(self._h)))
        self.n = mesh.num_nodes
        self.nnz = mesh.nnz

    def close(self):
        if self._h:
            N.lib().tg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        return N.check(rc, self._h)

    # Grid_3d::Table
    def relax(self, cycles: int) -> float:
        dev = C.c_double()
        self._ck(N.lib().tg_relax_cycles(self._h, cycles, C.byref(dev)))
        return dev.value

    def relax_threshold(self, threshold: float, cycle: int, queue: int, max_sweeps: int = 0):
        it, dev = C.c_int64(), C.c_double()
        rc = N.lib().tg_relax_threshold(self._h, threshold, cycle, queue, max_sweeps, C.byref(it), C.byref(dev))
        if rc not in (N.TG_OK, N.TG_ERR_RELAX_FAULT, N.TG_ERR_ITERATION_CAP):
            self._ck(rc)
        return rc, it.value, dev.value

    def local_relax(self, node: int, shell: int, threshold: float, cycle: int, queue: int):
        it, dev = C.c_int64(), C.c_double()
        rc = N.lib().tg_local_relax(self._h, node, shell, threshold, cycle, queue, C.byref(it), C.byref(dev))
        if rc not in (N.TG_OK, N.TG_ERR_RELAX_FAULT, N.TG_ERR_ITERATION_CAP):
            self._ck(rc)
        return rc, it.value, dev.value

    def solve(self, rel_tol=1e-8, max_outer=20, max_inner=4000, inner_rtol=1e-4, warm_start=0,
              preconditioner=0, inner_precision=0) -> N.tg_solve_info:
        info = N.tg_solve_info()
        o = solve_opts(rel_tol, max_outer, max_inner, inner_rtol, warm_start, preconditioner, inner_precision)
        self._ck(N.lib().tg_solve(self._h, C.byref(o), C.byref(info)))
        return info

    def set_launch_mode(self, mode: int):
        """2 (the default): the multigrid solve replays one captured CG
        iteration (a CUDA graph) inside a device-side loop; 1: replays it
        from the host in batches; 0: launches every kernel
        (tg_set_launch_mode)."""
        N.check(N.lib().tg_set_launch_mode(self._h, int(mode)), self._h)

    def amg_schedule(self) -> list[dict]:
        """Per multigrid level: rows and the tuned lanes per CSR row of its
        operator and restriction with their launch times (tg_amg_schedule)."""
        out = []
        level = 0
        while True:
            rows, al, rl = C.c_int32(), C.c_int32(), C.c_int32()
            am, rm = C.c_float(), C.c_float()
            rc = N.lib().tg_amg_schedule(self._h, level, C.byref(rows), C.byref(al), C.byref(rl), C.byref(am),
                                         C.byref(rm))
            if rc != N.TG_OK:
                if level == 0:
                    self._ck(rc)
                break
            out.append({"level": level, "rows": rows.value, "a_lanes": al.value, "r_lanes": rl.value,
                        "a_ms": am.value, "r_ms": rm.value})
            level += 1
        return out

    def residual(self) -> float:
        r = C.c_double()
        self._ck(N.lib().tg_residual(self._h, C.byref(r)))
        return r.value

    def potentials(self) -> np.ndarray:
        out = np.empty(self.n, np.float64)
        self._ck(N.lib().tg_get_phi(self._h, N.ptr(out)))
        return out

    def set_potentials(self, phi: np.ndarray):
        p = np.ascontiguousarray(phi, np.float64)
        self._ck(N.lib().tg_set_phi(self._h, N.ptr(p)))

    def field_o1(self, nodes) -> np.ndarray:
        nd = np.ascontiguousarray(np.atleast_1d(nodes), np.int32)
        out = np.empty((len(nd), 3), np.float64)
        self._ck(N.lib().tg_field_o1(self._h, len(nd), N.ptr(nd), N.ptr(out)))
        return out

    def couplings(self) -> np.ndarray:
        out = np.empty(self.nnz, np.float64)
        self._ck(N.lib().tg_get_couplings(self._h, N.ptr(out)))
        return out

    def types(self) -> np.ndarray:
        out = np.empty(self.n, np.int8)
        self._ck(N.lib().tg_get_types(self._h, N.ptr(out)))
        return out

    # Surface_3d
    def surface_init(self, vacuum_id: int) -> int:
        ns = C.c_int32()
        self._ck(N.lib().tg_surface_init(self._h, vacuum_id, C.byref(ns)))
        return ns.value

    def select(self, mode: int = 0, temperature: float = 0.0) -> N.tg_select_info:
        """Probabilities of probability mode `mode` (0 linear field, 1
        Boltzmann, 2 linear force, 3 Voronoi flux force) and evapMaximum's
        candidate."""
        info = N.tg_select_info()
        rc = N.lib().tg_surface_select_mode(self._h, mode, temperature, C.byref(info))
        if rc not in (N.TG_OK, N.TG_ERR_NO_SURFACE):
            self._ck(rc)
        return info

    def pick(self, u: float) -> tuple[int, float]:
        """evapMonteCarlo on the last selection for a uniform draw u."""
        node, p = C.c_int32(), C.c_float()
        self._ck(N.lib().tg_surface_pick(self._h, u, C.byref(node), C.byref(p)))
        return node.value, p.value

    def surface(self):
        cnt = C.c_int32()
        self._ck(N.lib().tg_get_surface(self._h, 0, None, None, C.byref(cnt)))
        nodes = np.empty(cnt.value, np.int32)
        ratios = np.empty(cnt.value, np.float32)
        self._ck(N.lib().tg_get_surface(self._h, cnt.value, N.ptr(nodes), N.ptr(ratios), C.byref(cnt)))
        order = np.argsort(nodes)
        return nodes[order], ratios[order]

    def cell_values(self, nodes=None, force: bool = True):
        """(phi, field [n, 3], force [n, 3] or None) as float of the listed
        cells, or of every cell (tg_cell_values)."""
        idx = None if nodes is None else np.ascontiguousarray(nodes, np.int32)
        n = self.n if idx is None else len(idx)
        phi = np.empty(n, np.float32)
        field = np.empty((n, 3), np.float32)
        frc = np.empty((n, 3), np.float32) if force else None
        self._ck(N.lib().tg_cell_values(self._h, n, N.ptr(idx), N.ptr(phi), N.ptr(field), N.ptr(frc)))
        return phi, field, frc

    def surface_normals(self, nodes) -> np.ndarray:
        idx = np.ascontiguousarray(nodes, np.int32)
        out = np.empty((len(idx), 3), np.float32)
        self._ck(N.lib().tg_surface_normals(self._h, len(idx), N.ptr(idx), N.ptr(out)))
        return out

    def surface_cells(self, mode: int = 0, temperature: float = 0.0):
        """(cells ascending, probabilities) of probability mode `mode`."""
        cnt = C.c_int32()
        self._ck(N.lib().tg_surface_cells(self._h, mode, temperature, 0, C.byref(cnt), None, None))
        cells = np.empty(cnt.value, np.int32)
        prob = np.empty(cnt.value, np.float32)
        self._ck(N.lib().tg_surface_cells(self._h, mode, temperature, cnt.value, C.byref(cnt), N.ptr(cells),
                                          N.ptr(prob)))
        return cells, prob

    def log_grid(self, path: str, index: int, binary: bool = False, numbers=None) -> str:
        """LogGrid snapshot of the current state into path.%08u; returns the name."""
        num = None if numbers is None else np.ascontiguousarray(numbers, np.uint32)
        self._ck(N.lib().tg_log_grid(self._h, str(path).encode(), index, int(binary), N.ptr(num)))
        return f"{path}.{index:08d}"

    def log_surface(self, path: str, index: int, binary: bool = False, with_neighbours: bool = False,
                    mode: int = 0, temperature: float = 0.0, numbers=None) -> str:
        """LogSurface snapshot of the current state into path.%08u."""
        num = None if numbers is None else np.ascontiguousarray(numbers, np.uint32)
        self._ck(N.lib().tg_log_surface(self._h, str(path).encode(), index, int(binary), int(with_neighbours), mode,
                                        temperature, N.ptr(num)))
        return f"{path}.{index:08d}"

    def normal(self, node: int) -> np.ndarray:
        out = np.empty(3, np.float32)
        self._ck(N.lib().tg_surface_normal(self._h, node, N.ptr(out)))
        return out

    def take_away(self, node: int) -> list[int]:
        cap = 256
        det = np.empty(cap, np.int32)
        nd = C.c_int32()
        self._ck(N.lib().tg_take_away(self._h, node, cap, N.ptr(det), C.byref(nd)))
        return det[: min(nd.value, cap)].tolist()

    def update_coordination(self):
        self._ck(N.lib().tg_update_coordination(self._h))

    # Trajectory_3d
    def trace(self, start: np.ndarray, qm, tet_guess=None, vel=None, **opts) -> np.ndarray:
        start = np.ascontiguousarray(np.atleast_2d(start), np.float32)
        n = len(start)
        q = np.ascontiguousarray(np.broadcast_to(np.asarray(qm, np.float32), (n,)))
        g = None if tet_guess is None else np.ascontiguousarray(np.broadcast_to(np.asarray(tet_guess, np.int32), (n,)))
        v = None if vel is None else np.ascontiguousarray(np.atleast_2d(vel), np.float32)
        out = (N.tg_impact * n)()
        self._ck(N.lib().tg_trace(self._h, n, N.ptr(start), N.ptr(v), N.ptr(q), N.ptr(g),
                                  C.byref(trace_opts(**opts)), C.cast(out, C.c_void_p)))
        return out

    def trace_path(self, start: np.ndarray, qm, tet_guess=None, vel=None, cap: int = 4096, **opts):
        """tg_trace_path: (impacts, paths, errors).  paths[k] is ion k's
        Trajectory_3d::data() as PATH_POINT records (start, accepted steps,
        extrapolated point; at most cap), errors[k] its error estimate
        (position x, y, z, velocity x, y, z)."""
        start = np.ascontiguousarray(np.atleast_2d(start), np.float32)
        n = len(start)
        q = np.ascontiguousarray(np.broadcast_to(np.asarray(qm, np.float32), (n,)))
        g = None if tet_guess is None else np.ascontiguousarray(np.broadcast_to(np.asarray(tet_guess, np.int32), (n,)))
        v = None if vel is None else np.ascontiguousarray(np.atleast_2d(vel), np.float32)
        out = (N.tg_impact * n)()
        pts = np.zeros((n, cap), N.PATH_POINT)
        err = np.zeros((n, 6), np.float32)
        self._ck(N.lib().tg_trace_path(self._h, n, N.ptr(start), N.ptr(v), N.ptr(q), N.ptr(g),
                                       C.byref(trace_opts(**opts)), cap, C.cast(out, C.c_void_p), N.ptr(pts),
                                       N.ptr(err)))
        return out, [pts[k, :path_length(out[k], cap)] for k in range(n)], err

    def potential_at(self, xyz: np.ndarray, tet_guess=None) -> np.ndarray:
        xyz = np.ascontiguousarray(np.atleast_2d(xyz), np.float32)
        g = None if tet_guess is None else np.ascontiguousarray(tet_guess, np.int32)
        out = np.empty(len(xyz), np.float32)
        self._ck(N.lib().tg_potential_at(self._h, len(xyz), N.ptr(xyz), N.ptr(g), N.ptr(out)))
        return out

    def run_event(self, opts: N.tg_event_opts, event_index: int) -> N.tg_event_record:
        rec = N.tg_event_record()
        self._ck(N.lib().tg_run_event(self._h, C.byref(opts), event_index, C.byref(rec)))
        return rec

    def run_events(self, opts: N.tg_event_opts, first_index: int, count: int) -> list:
        """`count` events in one call, flights overlapping the next event's
        relaxation (tg_run_events); returns the records."""
        recs = (N.tg_event_record * count)()
        done = C.c_int32()
        rc = N.lib().tg_run_events(self._h, C.byref(opts), first_index, count, C.cast(recs, C.c_void_p),
                                   C.byref(done))
        self._ck(rc)
        return list(recs)[:done.value]


class Learner:
    """The learned near-field warm start (tg_learner_*): a message-passing
    network on the free cells within `hops` steps of each removed atom,
    trained on the device from samples that `Grid.solve` collects."""

    def __init__(self, hops: int = 6, max_cells: int = 4096, ell_width: int = 64, seed: int = 1):
        self._h = C.c_void_p()
        N.check(N.lib().tg_learner_create(hops, max_cells, ell_width, seed, C.byref(self._h)))
        self.ell_width = ell_width
        self.num_params = int(N.lib().tg_learner_num_params())

    def close(self):
        if self._h:
            N.lib().tg_learner_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        if rc != N.TG_OK:
            msg = N.lib().tg_learner_last_error(self._h)
            raise N.TapsimError(rc, msg.decode() if msg else "")
        return rc

    def attach(self, grid: "Grid", collect: bool = False, predict: bool = False):
        """Attach to a grid: collect samples in its event solves and/or add
        the prediction to solves with warm_start=2."""
        mode = (1 if collect else 0) | (2 if predict else 0)
        grid._ck(N.lib().tg_learner_attach(grid._h, self._h if mode else None, mode))

    def set_gain(self, gain: float):
        """Multiplier of the prediction that warm_start=2 adds (default 1;
        0: no prediction, the refinement sweeps alone)."""
        self._ck(N.lib().tg_learner_set_gain(self._h, gain))

    def set_refine(self, sweeps: int):
        """Damped Jacobi sweeps over the prediction's cells after it (tg_learner_set_refine)."""
        self._ck(N.lib().tg_learner_set_refine(self._h, sweeps))

    def samples(self) -> tuple[int, int]:
        n, cells = C.c_int32(), C.c_int64()
        self._ck(N.lib().tg_learner_samples(self._h, C.byref(n), C.byref(cells)))
        return n.value, cells.value

    def params(self) -> np.ndarray:
        out = np.empty(self.num_params, np.float32)
        self._ck(N.lib().tg_learner_get_params(self._h, N.ptr(out)))
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.num_params
        self._ck(N.lib().tg_learner_set_params(self._h, N.ptr(p)))

    def sample(self, idx: int) -> dict:
        n = C.c_int32()
        self._ck(N.lib().tg_learner_get_sample(self._h, idx, C.byref(n), None, None, None, None))
        k = n.value
        X = np.empty((k, 16), np.float32)
        col = np.empty((k, self.ell_width), np.int32)
        w = np.empty((k, self.ell_width), np.float32)
        t = np.empty(k, np.float32)
        self._ck(N.lib().tg_learner_get_sample(self._h, idx, C.byref(n), N.ptr(X), N.ptr(col), N.ptr(w), N.ptr(t)))
        return {"X": X, "col": col, "w": w, "target": t}

    def gradients(self, first: int, count: int = 1):
        """(loss, gradient, outputs) over samples first..first+count-1."""
        rows = sum(self.sample(k)["target"].size for k in range(first, first + count))
        loss = C.c_float()
        g = np.empty(self.num_params, np.float32)
        y = np.empty(rows, np.float32)
        self._ck(N.lib().tg_learner_gradients(self._h, first, count, C.byref(loss), N.ptr(g), N.ptr(y)))
        return loss.value, g, y

    def train(self, steps: int, batch: int = 8, lr: float = 1e-3, seed: int = 0, first: int = 0,
              count: int = 0) -> float:
        loss = C.c_float()
        self._ck(N.lib().tg_learner_train(self._h, steps, batch, lr, seed, first, count, C.byref(loss)))
        return loss.value


# ---- tapsim.ini -----------------------------------------------------------

# Process::EvaporationOptions keys (process.cpp:206-439) with the internal
# defaults of makeIniList (commands.cpp:1249-1325)
INI_DEFAULTS = {
    "RESULTS_FILENAME": "results_data", "RESULTS_BINARY_OUTPUT": "0", "RESULTS_CHUNK_SIZE": "10000",
    "TRAJECTORY_FILENAME": "trajectory_data", "TRAJECTORY_BINARY_OUTPUT": "1", "TRAJECTORY_CHUNK_SIZE": "10000",
    "GRID_FILENAME": "grid_data", "GRID_BINARY_OUTPUT": "1", "GRID_INTERVAL": "2147483647",
    "SURFACE_FILENAME": "surface_data", "SURFACE_BINARY_OUTPUT": "1", "SURFACE_INTERVAL": "2147483647",
    "GEOMETRY_FILENAME": "geometry.dat", "GEOMETRY_BINARY_OUTPUT": "1", "GEOMETRY_CONTENTS": "0xff",
    "DUMP_FILENAME": "dump", "DUMP_INTERVAL": "10000", "OUTPUT_DELAY_TIME": "60",
    "METHOD_EVAPORATION_PROBABILITY": "0", "METHOD_EVAPORATION_CHOICE": "0", "VACUUM_CELL_IDENTIFIER": "Vacuum",
    "TRAJECTORY_INTEGRATOR_TYPE": "1", "TRAJECTORY_STEPPER_TYPE": "1", "TRAJECTORY_INITIAL_TIME_STEP": "1e-14",
    "TRAJECTORY_MINIMUM_TIME_STEP": "1e-16", "TRAJECTORY_ERROR_THRESHOLD": "1e-6",
    "TRAJECTORY_NON_RANDOM_START_POSITION": "1", "TRAJECTORY_NO_INITIAL_VELOCITY": "1",
    "VOLTAGE_QUEUE_SIZE": "250", "LOCAL_RELAXATION_ERROR_THRESHOLD": "1e-2", "LOCAL_RELAXATION_SHELL_SIZE": "3",
    "LOCAL_RELAXATION_CYCLE_SIZE": "5", "LOCAL_RELAXATION_QUEUE_SIZE": "5", "GLOBAL_RELAXATION_STEPS": "1",
    "REFRESH_RELAXATION_INTERVAL": "0", "REFRESH_RELAXATION_ERROR_THRESHOLD": "0.0",
    "REFRESH_RELAXATION_CYCLE_SIZE": "100", "REFRESH_RELAXATION_QUEUE_SIZE": "25",
}


def read_ini(path: str | None) -> dict:
    """File_Io::readInitialization: 'KEY = VALUE' lines, '#' comments, unique keys."""
    if path is None:
        return dict(INI_DEFAULTS)
    values = {}
    for line in Path(path).read_text().splitlines():
        if not line or line.startswith("#"):
            continue
        if " = " not in line:
            raise ValueError(f"ini: bad line {line!r}")
        k, v = line.split(" = ", 1)
        k, v = k.strip(), v.strip()
        if k in values:
            raise ValueError(f"ini: duplicate key {k}")
        values[k] = v
    return values


@dataclass
class EvaporationOptions:
    values: dict = field(default_factory=lambda: dict(INI_DEFAULTS))

    @classmethod
    def from_ini(cls, path: str | None) -> "EvaporationOptions":
        v = read_ini(path)
        missing = [k for k in INI_DEFAULTS if k not in v]
        if missing:
            # setDefaults throws on the first missing key
            raise ValueError(f"EvaporationOptions::setDefaults(): '{missing[0]}' error!")
        return cls(v)

    def i(self, k):
        return int(self.values[k], 0) if k == "GEOMETRY_CONTENTS" else int(float(self.values[k]))

    def f(self, k):
        return float(self.values[k])

    def s(self, k):
        return self.values[k]

    def event_opts(self, vacuum_id: int, relax_mode: int, solve: N.tg_solve_opts | None = None,
                   trace: bool = True, normal: bool = True, refresh_max_sweeps: int = 2_000_000,
                   temperature: float = 0.0, rng_seed: int = 99) -> N.tg_event_opts:
        o = N.tg_event_opts()
        o.prob_mode = self.i("METHOD_EVAPORATION_PROBABILITY")
        o.choice_mode = self.i("METHOD_EVAPORATION_CHOICE")
        o.temperature = temperature
        o.rng_seed = rng_seed
        o.vacuum_id = vacuum_id
        o.relax_mode = relax_mode
        o.local_threshold = self.f("LOCAL_RELAXATION_ERROR_THRESHOLD")
        o.local_shell = self.i("LOCAL_RELAXATION_SHELL_SIZE")
        o.local_cycle = self.i("LOCAL_RELAXATION_CYCLE_SIZE")
        o.local_queue = self.i("LOCAL_RELAXATION_QUEUE_SIZE")
        o.global_steps = self.i("GLOBAL_RELAXATION_STEPS")
        o.refresh_interval = self.i("REFRESH_RELAXATION_INTERVAL")
        o.refresh_threshold = self.f("REFRESH_RELAXATION_ERROR_THRESHOLD")
        o.refresh_cycle = self.i("REFRESH_RELAXATION_CYCLE_SIZE")
        o.refresh_queue = self.i("REFRESH_RELAXATION_QUEUE_SIZE")
        o.refresh_max_sweeps = refresh_max_sweeps
        o.solve = solve if solve is not None else solve_opts()
        o.trace = trace_opts(self.f("TRAJECTORY_INITIAL_TIME_STEP"), self.f("TRAJECTORY_MINIMUM_TIME_STEP"),
                             self.f("TRAJECTORY_ERROR_THRESHOLD"), integrator=self.i("TRAJECTORY_INTEGRATOR_TYPE"),
                             stepper=self.i("TRAJECTORY_STEPPER_TYPE"))
        o.initial_velocity = 0 if self.i("TRAJECTORY_NO_INITIAL_VELOCITY") else 1
        o.trace_enabled = int(trace)
        o.normal_enabled = int(normal)
        return o


# ---- event loop -------------------------------------------------------------

RESULT_FIELDS = ["index", "id", "number", "voltage", "startX", "startY", "startZ", "stopX", "stopY", "stopZ", "tof",
                 "probability", "potentialBefore", "fieldBeforeX", "fieldBeforeY", "fieldBeforeZ", "potentialAfter",
                 "fieldAfterX", "fieldAfterY", "fieldAfterZ", "normalX", "normalY", "normalZ", "apexX", "apexY",
                 "apexZ"]


class Evaporation:
    """Process::evaporation (process.cpp:441-1124) over one device Grid."""

    def __init__(self, grid: Grid, options: EvaporationOptions, relax_mode: int = 1,
                 solve: N.tg_solve_opts | None = None, trace: bool = True, normal: bool = True, path_cap: int = 0,
                 snapshots: bool = False):
        """path_cap > 0 keeps each event's flight path (up to path_cap points)
        in its record for write_trajectories.  snapshots writes the grid and
        surface snapshots that GRID_FILENAME / SURFACE_FILENAME, *_INTERVAL
        and *_BINARY_OUTPUT ask for (process.cpp:641-643, 1068-1072): once
        before the first event and after every event whose index is a
        multiple of the interval."""
        self.grid = grid
        self.options = options
        types = grid.mesh.arrays()["types"]
        name = options.s("VACUUM_CELL_IDENTIFIER")
        self.vacuum_id = self._type_id_by_name(grid, name)
        self.evap_field = {k: v["evap_field"] for k, v in types.items()}
        # the ion's charge [C] and mass [kg] as Process::evaporation forms
        # them in float (process.cpp:929-933)
        self.charge_mass = {k: (float(np.float32(v["evap_charge"]) * np.float32(1.60217733e-19)),
                                float(np.float32(v["mass"]) * np.float32(1.660538782e-27))) for k, v in types.items()}
        self.path_cap = int(path_cap)
        self.numbers = grid.mesh.numbers()
        self.snapshots = bool(snapshots)
        self.opts = options.event_opts(self.vacuum_id, relax_mode, solve, trace, normal,
                                       temperature=grid.mesh.temperature)
        self.voltage_queue: deque = deque()
        self.voltage_sum = 0.0
        self.queue_size = options.i("VOLTAGE_QUEUE_SIZE")
        self.event = 0
        self.records: list[dict] = []
        grid.surface_init(self.vacuum_id)
        grid.select()
        if self.snapshots:
            self._snapshot(force=True)

    def _snapshot_logs(self):
        for key in ("GRID", "SURFACE"):
            name = self.options.s(f"{key}_FILENAME")
            if name:
                yield key, name, self.options.i(f"{key}_INTERVAL"), self.options.i(f"{key}_BINARY_OUTPUT") != 0

    def _snapshot(self, force: bool = False):
        """Step VII's snapshots (process.cpp:1068-1072) after event self.event."""
        for key, name, interval, binary in self._snapshot_logs():
            if not force and (interval <= 0 or self.event % interval != 0):
                continue
            if key == "GRID":
                self.grid.log_grid(name, self.event, binary, self.numbers)
            else:
                self.grid.log_surface(name, self.event, binary, False, self.opts.prob_mode, self.opts.temperature,
                                      self.numbers)

    def _events_to_snapshot(self) -> int:
        """Events until the next one after which a snapshot is due."""
        k = 1 << 62
        if self.snapshots:
            for _, _, interval, _ in self._snapshot_logs():
                if interval > 0:
                    k = min(k, interval - self.event % interval)
        return k

    @staticmethod
    def _type_id_by_name(grid: Grid, name: str) -> int:
        names = getattr(grid.mesh, "type_names", None)
        if names and name in names:
            return names[name]
        # meshgen's vacuum marker is id 0 in every generated configuration
        return 0

    def _path_buffers(self, count: int):
        if self.path_cap <= 0:
            self.opts.path_cap = 0
            self.opts.path_points = None
            self.opts.path_errors = None
            return None, None
        pts = np.zeros((count, self.path_cap), N.PATH_POINT)
        err = np.zeros((count, 6), np.float32)
        self.opts.path_cap = self.path_cap
        self.opts.path_points = pts.ctypes.data
        self.opts.path_errors = err.ctypes.data
        return pts, err

    def step(self) -> dict:
        self.event += 1
        pts, err = self._path_buffers(1)
        rec = self.grid.run_event(self.opts, self.event)
        r = self._record(rec, None if pts is None else (pts[0], err[0]))
        self.records.append(r)
        if self.snapshots:
            self._snapshot()
        return r

    def run(self, count: int, force=None) -> list[dict]:
        """`count` events in one library call: each ion flight overlaps the
        next event's removal and relaxation.  Same records as `step`.
        force: node indices that the first len(force) events remove in place
        of the chosen cells (tg_event_opts.force_nodes); a record whose
        probability is below its best_probability removed a forced cell
        that was not this run's choice."""
        out = []
        forced = None if force is None else np.ascontiguousarray(force, np.int32)
        done = 0
        while count > 0:
            # a batch ends where a snapshot is due
            k = min(count, self._events_to_snapshot())
            pts, err = self._path_buffers(k)
            if forced is not None and done < len(forced):
                self.opts.force_nodes = forced[done:].ctypes.data
                self.opts.force_count = len(forced) - done
            else:
                self.opts.force_nodes = None
                self.opts.force_count = 0
            recs = self.grid.run_events(self.opts, self.event + 1, k)
            done += k
            for j, rec in enumerate(recs):
                self.event += 1
                r = self._record(rec, None if pts is None else (pts[j], err[j]))
                self.records.append(r)
                out.append(r)
            if self.snapshots:
                self._snapshot()
            count -= k
        return out

    def _record(self, rec: N.tg_event_record, path=None) -> dict:
        """Step VI: voltage queue and time-of-flight scale (process.cpp:985-1036)."""
        imp = rec.impact
        # in float, operation by operation, as process.cpp:985-1036 does
        f32 = np.float32
        fbv = [f32(x) for x in rec.field_before]
        fb = f32(np.sqrt(fbv[0] * fbv[0] + fbv[1] * fbv[1] + fbv[2] * fbv[2]))
        if imp.last_tet >= 0 and fb != 0.0:
            v = f32(rec.phi_before) - f32(imp.last_phi)
            v = v * f32(self.evap_field[rec.type_id])
            v = v / fb
            v = v / f32(rec.scaling_reference)
            self.voltage_queue.append(v)
            self.voltage_sum = f32(self.voltage_sum + v)
            while len(self.voltage_queue) > self.queue_size:
                self.voltage_sum = f32(self.voltage_sum - self.voltage_queue.popleft())
            voltage = f32(self.voltage_sum / f32(len(self.voltage_queue)))
            ts = (f32(rec.phi_after) - f32(imp.last_phi)) / voltage
            with np.errstate(invalid="ignore"):
                time_scale = float(np.sqrt(f32(ts)))
            voltage = float(voltage)
        else:
            voltage = 1.0 if fb == 0.0 else 0.0
            time_scale = 1.0
        return {
            "index": self.event, "node": rec.node, "id": rec.type_id, "number": int(self.numbers[rec.node]),
            "voltage": voltage,
            "stop": tuple(imp.stop), "tof": float(np.float32(imp.stop_time) * np.float32(time_scale)),
            "probability": rec.probability,
            "best": rec.best_ratio, "second": rec.second_ratio, "scaling_reference": rec.scaling_reference,
            "potentialBefore": rec.phi_before, "fieldBefore": tuple(rec.field_before),
            "potentialAfter": rec.phi_after, "fieldAfter": tuple(rec.field_after), "normal": tuple(rec.normal),
            "apex": tuple(rec.apex), "status": imp.status, "steps": imp.steps, "detached": rec.detached,
            "relax_iterations": rec.relax_iterations, "rel_residual": rec.rel_residual,
            "best_probability": rec.best_probability, "second_probability": rec.second_probability,
            "time_scale": time_scale, "charge": self.charge_mass[rec.type_id][0],
            "mass": self.charge_mass[rec.type_id][1],
        } | ({} if path is None else {"path": path[0][:path_length(imp, self.path_cap)].copy(),
                                      "path_error": path[1].copy()})


def _chunk_names(path: str, indices: list, chunk_size: int) -> list:
    """The files a chunked log writes: path.%08u after the index opening
    each chunk (a new chunk when index % chunk_size == 0), else path."""
    if chunk_size <= 0 or not indices:
        return [path]
    return [f"{path}.{i:08d}" for k, i in enumerate(indices) if k == 0 or i % chunk_size == 0]


def write_results_rows(path: str, rows: list, binary: bool = False, header: str = "", chunk_size: int = 0) -> list:
    """Results files in LogResults' layout (logResults.cpp:135-381) from rows
    of the 26 RESULT_FIELDS values, by the library's native writer
    (tg_results_write).  With chunk_size > 0 the rows go to files named
    path.%08u after the index of the event opening each chunk, the header
    only in the first, as the reference's writer thread does.  Returns the
    file names."""
    arr = (N.tg_result_row * len(rows))()
    for k, r in enumerate(rows):
        a = arr[k]
        a.index, a.id, a.number, a.voltage = int(r[0]), int(r[1]), int(r[2]), float(r[3])
        a.start[:] = [float(v) for v in r[4:7]]
        a.stop[:] = [float(v) for v in r[7:10]]
        a.tof, a.probability, a.potential_before = float(r[10]), float(r[11]), float(r[12])
        a.field_before[:] = [float(v) for v in r[13:16]]
        a.potential_after = float(r[16])
        a.field_after[:] = [float(v) for v in r[17:20]]
        a.normal[:] = [float(v) for v in r[20:23]]
        a.apex[:] = [float(v) for v in r[23:26]]
    N.check(N.lib().tg_results_write(str(path).encode(), int(binary), header.encode(), len(rows),
                                     C.cast(arr, C.c_void_p), int(chunk_size)))
    return _chunk_names(str(path), [int(r[0]) for r in rows], chunk_size)


def read_results(path: str) -> tuple[str, list]:
    """(header, rows) of one results file, ASCII or binary."""
    data = open(path, "rb").read()
    lines = data.split(b"\n")
    head, k = [], 2
    while not lines[k].startswith(b"# index"):
        head.append(lines[k].decode() + "\n")
        k += 1
    k += len(RESULT_FIELDS)
    mode = lines[k]
    body_start = sum(len(l) + 1 for l in lines[:k + 1])
    rows = []
    if mode == b"BINARY":
        rec = struct.Struct("<IhI23f")
        body = data[body_start:]
        for o in range(0, len(body) - len(body) % rec.size, rec.size):
            rows.append(list(rec.unpack_from(body, o)))
    else:
        for l in lines[k + 1:]:
            if l.strip():
                t = l.decode().split("\t")
                rows.append([int(t[0]), int(t[1]), int(t[2])] + [float(x) for x in t[3:]])
    return "".join(head), rows


def write_results(path: str, records: list[dict], xyz: np.ndarray, binary: bool = False, header: str = "",
                  chunk_size: int = 0) -> list:
    """Results files of Evaporation records (LogResults::Dataset,
    logResults.h:41-66)."""
    rows = []
    for r in records:
        start = xyz[r["node"]]
        rows.append([r["index"], r["id"], r["number"], r["voltage"], *start, *r["stop"], r["tof"],
                     r["probability"], r["potentialBefore"], *r["fieldBefore"], r["potentialAfter"],
                     *r["fieldAfter"], *r["normal"], *r["apex"]])
    return write_results_rows(path, rows, binary, header, chunk_size)

# ---- trajectory files (LogTrajectory) -----------------------------------------

def write_trajectory_items(path: str, items: list, binary: bool = False, chunk_size: int = 0) -> list:
    """Trajectory files in LogTrajectory's layout (logTrajectory.cpp:170-300)
    by the library's native writer (tg_trajectory_write).  Each item holds
    index, number, time_scale, status, charge, mass, points (PATH_POINT
    records whose time column is written as it is) and error (6 floats).
    With chunk_size > 0 the items go to files named path.%08u after the index
    opening each chunk, each file with the header.  Returns the file names."""
    arr = (N.tg_trajectory_item * len(items))()
    keep = []
    for k, it in enumerate(items):
        pts = np.ascontiguousarray(np.asarray(it["points"], N.PATH_POINT))
        keep.append(pts)
        a = arr[k]
        a.index, a.number, a.time_scale, a.status = int(it["index"]), int(it["number"]), float(it["time_scale"]), \
            int(it["status"])
        a.charge, a.mass, a.num_points = float(it["charge"]), float(it["mass"]), len(pts)
        a.points = pts.ctypes.data if len(pts) else None
        a.error[:] = [float(v) for v in it["error"]]
    N.check(N.lib().tg_trajectory_write(str(path).encode(), int(binary), len(items), C.cast(arr, C.c_void_p),
                                        int(chunk_size)))
    return _chunk_names(str(path), [int(it["index"]) for it in items], chunk_size)


def write_trajectories(path: str, records: list[dict], binary: bool = False, chunk_size: int = 0) -> list:
    """Trajectory files of Evaporation records kept with path_cap > 0
    (Process::evaporation step VII, process.cpp:1048-1049): each point's
    time is written times the event's time scale, in float."""
    items = []
    for r in records:
        if "path" not in r:
            raise ValueError("write_trajectories: records carry no path (Evaporation(..., path_cap=...))")
        pts = r["path"].copy()
        pts["time"] = pts["time"] * np.float32(r["time_scale"])
        items.append({"index": r["index"], "number": r["number"], "time_scale": r["time_scale"],
                      "status": r["status"], "charge": r["charge"], "mass": r["mass"], "points": pts,
                      "error": r["path_error"]})
    return write_trajectory_items(path, items, binary, chunk_size)


def read_trajectories(path: str) -> tuple[bool, list]:
    """(binary, items) of one trajectory file, items as
    write_trajectory_items takes them."""
    data = open(path, "rb").read()
    pos = data.index(b"\n\n") + 2  # header ends with an empty line
    binary = b"(float)" in data[:pos]
    items = []

    def line():
        nonlocal pos
        end = data.index(b"\n", pos)
        out = data[pos:end].decode()
        pos = end + 1
        return out

    def value(text):
        return text.split(" = ", 1)[1]

    while pos < len(data):
        index = int(value(line()))
        number = int(value(line()))
        ts = float(value(line()))
        status = int(value(line()).split(" => ")[0])
        charge, mass = (float(x) for x in value(line()).split(" / "))
        mode, count = line().split(" ")
        count = int(count)
        if mode == "BINARY":
            pts = np.frombuffer(data, N.PATH_POINT, count, pos).copy()
            pos += count * N.PATH_POINT.itemsize + 1
        else:
            pts = np.zeros(count, N.PATH_POINT)
            for k in range(count):
                t = line().split("\t")
                pts[k] = (float(t[0]), [float(x) for x in t[1:4]], [float(x) for x in t[4:7]], int(t[7]))
        err = []
        for _ in range(2):
            err += [float(x) for x in value(line()).strip("()").split("/")]
        line()  # the empty line after each trajectory
        items.append({"index": index, "number": number, "time_scale": ts, "status": status, "charge": charge,
                      "mass": mass, "points": pts, "error": np.array(err, np.float32)})
    return binary, items


# ---- grid and surface snapshots (LogGrid, LogSurface) --------------------------

GRID_RECORD = np.dtype([("id", "<i2"), ("number", "<u4"), ("phi", "<f4"), ("field", "<f4", 3), ("force", "<f4", 3)],
                       align=False)


def write_grid_log(path: str, id, number, phi, field, force, binary: bool = False):
    """One grid snapshot file in LogGrid's layout (logGrid.cpp:197-245),
    written by the library's native writer."""
    id = np.ascontiguousarray(id, np.int32)
    n = len(id)
    arrs = [np.ascontiguousarray(number, np.uint32), np.ascontiguousarray(phi, np.float32),
            np.ascontiguousarray(np.reshape(field, (n, 3)), np.float32),
            np.ascontiguousarray(np.reshape(force, (n, 3)), np.float32)]
    N.check(N.lib().tg_grid_log_write(str(path).encode(), int(binary), n, N.ptr(id), *[N.ptr(a) for a in arrs]))


def read_grid_log(path: str) -> tuple[bool, np.ndarray]:
    """(binary, records GRID_RECORD) of one grid snapshot file."""
    data = open(path, "rb").read()
    head = data.split(b"\n", 3)
    mode, count = head[2].decode().split(" ")
    count = int(count)
    body = head[3]
    if mode == "BINARY":
        return True, np.frombuffer(body, GRID_RECORD, count).copy()
    out = np.zeros(count, GRID_RECORD)
    rows = [l.split(b"\t") for l in body.split(b"\n")[:count]]
    out["id"] = [int(r[0]) for r in rows]
    out["number"] = [int(r[1]) for r in rows]
    vals = np.array([[float(x) for x in r[2:9]] for r in rows], np.float32).reshape(count, 7)
    out["phi"] = vals[:, 0]
    out["field"] = vals[:, 1:4]
    out["force"] = vals[:, 4:7]
    return False, out


def write_surface_log(path: str, cells: dict, nodes: dict, binary: bool = False):
    """One surface snapshot file in LogSurface's layout
    (logSurface.cpp:203-293), written by the library's native writer.
    cells: index, type, number, probability and optionally neighbours (a
    list of arrays); nodes: index, phi, field [n, 3], normal [n, 3]."""
    ci = np.ascontiguousarray(cells["index"], np.int32)
    ct = np.ascontiguousarray(cells["type"], np.int32)
    cn = np.ascontiguousarray(cells["number"], np.uint32)
    cp = np.ascontiguousarray(cells["probability"], np.float32)
    nptr = nb = None
    if cells.get("neighbours") is not None:
        lens = [len(x) for x in cells["neighbours"]]
        nptr = np.ascontiguousarray(np.concatenate([[0], np.cumsum(lens)]), np.int32)
        nb = np.ascontiguousarray(np.concatenate([np.asarray(x, np.int32) for x in cells["neighbours"]] or
                                                 [np.zeros(0, np.int32)]), np.int32)
    ni = np.ascontiguousarray(nodes["index"], np.int32)
    nphi = np.ascontiguousarray(nodes["phi"], np.float32)
    nf = np.ascontiguousarray(np.reshape(nodes["field"], (len(ni), 3)), np.float32)
    nn = np.ascontiguousarray(np.reshape(nodes["normal"], (len(ni), 3)), np.float32)
    N.check(N.lib().tg_surface_log_write(str(path).encode(), int(binary), len(ci), N.ptr(ci), N.ptr(ct), N.ptr(cn),
                                         N.ptr(cp), N.ptr(nptr), N.ptr(nb), len(ni), N.ptr(ni), N.ptr(nphi),
                                         N.ptr(nf), N.ptr(nn)))


def read_surface_log(path: str) -> tuple[bool, dict, dict]:
    """(binary, cells, nodes) of one surface snapshot file; cells carry
    "neighbours" (list of arrays, empty when the file has none)."""
    data = open(path, "rb").read()
    binary = data.split(b"\n")[2] == b"BINARY"
    pos = data.index(b"CELLS ")
    end = data.index(b"\n", pos)
    nc = int(data[pos + 6:end])
    pos = end + 1
    cells = {"index": np.zeros(nc, np.int32), "type": np.zeros(nc, np.int32), "number": np.zeros(nc, np.uint32),
             "probability": np.zeros(nc, np.float32), "neighbours": []}
    if binary:
        for c in range(nc):
            idx, typ, num, prob, cnt = struct.unpack_from("<ihIfI", data, pos)
            pos += 18
            nbrs = np.frombuffer(data, "<i4", cnt, pos).copy()
            pos += 4 * cnt
            cells["index"][c], cells["type"][c], cells["number"][c], cells["probability"][c] = idx, typ, num, prob
            cells["neighbours"].append(nbrs)
        pos += 1  # the newline after the cells
    else:
        for c in range(nc):
            end = data.index(b"\n", pos)
            t = data[pos:end].split(b"\t")
            pos = end + 1
            cells["index"][c], cells["type"][c], cells["number"][c] = int(t[0]), int(t[1]), int(t[2])
            cells["probability"][c] = float(t[3])
            cells["neighbours"].append(np.array([int(x) for x in t[5:]], np.int32) if len(t) > 4 else
                                       np.zeros(0, np.int32))
        pos += 1  # the empty line
    end = data.index(b"\n", pos)
    assert data[pos:pos + 6] == b"NODES "
    nn = int(data[pos + 6:end])
    pos = end + 1
    if binary:
        rec = np.dtype([("index", "<i4"), ("phi", "<f4"), ("field", "<f4", 3), ("normal", "<f4", 3)])
        arr = np.frombuffer(data, rec, nn, pos)
        nodes = {"index": arr["index"].copy(), "phi": arr["phi"].copy(), "field": arr["field"].copy(),
                 "normal": arr["normal"].copy()}
    else:
        rows = [l.split(b"\t") for l in data[pos:].split(b"\n")[:nn]]
        vals = np.array([[float(x) for x in r[1:8]] for r in rows], np.float32).reshape(nn, 7)
        nodes = {"index": np.array([int(r[0]) for r in rows], np.int32), "phi": vals[:, 0], "field": vals[:, 1:4],
                 "normal": vals[:, 4:7]}
    if not any(len(x) for x in cells["neighbours"]) and not binary:
        cells["neighbours"] = None
    return binary, cells, nodes
