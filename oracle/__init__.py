"""Test oracle: FP64 CPU restatement of TAPSim's per-event hot path.

Test infrastructure only.  tests/, __graft_entry__.smoke() and the CPU leg of
bench.py use it as the checker; nothing in tapsim_modified_b200 imports it.
The C code is in tapsim_oracle.c (built by `make -C oracle oracle`); the
reference built from its own sources (`make -C oracle ref`, outputs in
oracle/_ref/) pins it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"


def build():
    subprocess.run(["make", "-C", str(HERE), "oracle"], check=True, capture_output=True)


class orc_type(C.Structure):
    _fields_ = [("present", C.c_int32), ("removable", C.c_int32), ("neumann", C.c_int32), ("dirichlet", C.c_int32),
                ("epsilon", C.c_double), ("evap_field", C.c_double), ("charge_density", C.c_double),
                ("phi", C.c_double), ("mass", C.c_double), ("evap_charge", C.c_int32),
                ("evap_energy", C.c_double)]


class orc_mesh(C.Structure):
    _fields_ = [("n", C.c_int32), ("xyz", C.c_void_p), ("type", C.c_void_p), ("hull", C.c_void_p),
                ("row_ptr", C.c_void_p), ("col", C.c_void_p), ("c", C.c_void_p), ("geom", C.c_void_p),
                ("area_pos", C.c_void_p), ("phi", C.c_void_p), ("q", C.c_void_p), ("volume", C.c_void_p),
                ("ntets", C.c_int32), ("tet_v", C.c_void_p), ("tet_n", C.c_void_p), ("types", C.c_void_p),
                ("surface", C.c_void_p)]


class orc_select_info(C.Structure):
    _fields_ = [("candidate", C.c_int32), ("apex", C.c_int32), ("num_surface", C.c_int32), ("best", C.c_float),
                ("second", C.c_float), ("sum", C.c_double)]


class orc_impact(C.Structure):
    _fields_ = [("stop", C.c_double * 3), ("stop_time", C.c_double), ("last_pos", C.c_double * 3),
                ("last_tet", C.c_int32), ("last_phi", C.c_double), ("steps", C.c_int32), ("status", C.c_int32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        P = C.POINTER(orc_mesh)
        L.orc_residual.restype = C.c_double
        L.orc_residual.argtypes = [P]
        L.orc_solve.restype = C.c_int64
        L.orc_solve.argtypes = [P, C.c_double, C.c_int64, C.c_double, C.POINTER(C.c_double)]
        L.orc_relax_cycles.restype = C.c_double
        L.orc_relax_cycles.argtypes = [P, C.c_int32]
        L.orc_field_o1.restype = C.c_int
        L.orc_field_o1.argtypes = [P, C.c_int32, C.c_void_p]
        L.orc_force.restype = None
        L.orc_force.argtypes = [P, C.c_int32, C.c_void_p]
        L.orc_surface_init.restype = C.c_int32
        L.orc_surface_init.argtypes = [P, C.c_int32]
        L.orc_select.restype = None
        L.orc_select.argtypes = [P, C.c_void_p, C.POINTER(orc_select_info)]
        L.orc_select_mode.restype = None
        L.orc_select_mode.argtypes = [P, C.c_int32, C.c_double, C.c_void_p, C.POINTER(orc_select_info)]
        L.orc_field_o2.restype = C.c_int
        L.orc_field_o2.argtypes = [P, C.c_int32, C.c_void_p, C.POINTER(C.c_double)]
        L.orc_score.restype = C.c_double
        L.orc_score.argtypes = [P, C.c_int32, C.c_int32, C.c_double]
        L.orc_pick.restype = C.c_int32
        L.orc_pick.argtypes = [P, C.c_void_p, C.c_double, C.c_double]
        L.orc_take_away.restype = C.c_int32
        L.orc_take_away.argtypes = [P, C.c_int32, C.c_int32, C.c_void_p, C.c_int32]
        L.orc_update_coordination.restype = None
        L.orc_update_coordination.argtypes = [P]
        L.orc_trace.restype = None
        L.orc_trace.argtypes = [P, C.c_void_p, C.c_double, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_int32,
                                C.c_int32, C.c_double, C.POINTER(orc_impact)]
        L.orc_trace_ext.restype = None
        L.orc_trace_ext.argtypes = [P, C.c_void_p, C.c_void_p, C.c_double, C.c_int32, C.c_double, C.c_double,
                                    C.c_double, C.c_int32, C.c_int32, C.c_double, C.c_int32, C.c_int32,
                                    C.POINTER(orc_impact)]
        L.orc_trace_path.restype = None
        L.orc_trace_path.argtypes = [P, C.c_void_p, C.c_void_p, C.c_double, C.c_int32, C.c_double, C.c_double,
                                     C.c_double, C.c_int32, C.c_int32, C.c_double, C.c_int32, C.c_int32,
                                     C.POINTER(orc_impact), C.c_int32, C.c_void_p, C.c_void_p]
        L.orc_potential_at.restype = C.c_double
        L.orc_potential_at.argtypes = [P, C.c_void_p, C.c_int32]
        L.orc_local_set.restype = C.c_int32
        L.orc_local_set.argtypes = [P, C.c_int32, C.c_int32, C.c_void_p, C.c_int32]
        L.orc_local_solve.restype = C.c_int64
        L.orc_local_solve.argtypes = [P, C.c_void_p, C.c_int32, C.c_double, C.c_int64]
        L.orc_stagnated.restype = C.c_int32
        L.orc_stagnated.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Oracle:
    """Mutable CPU copy of a mesh description (dict from tapsim Mesh.arrays())."""

    def __init__(self, arrays: dict):
        a = arrays
        n = len(a["type"])
        self.n = n
        self.xyz = np.ascontiguousarray(a["xyz"], np.float32).reshape(-1)
        self.type = np.ascontiguousarray(a["type"], np.int8).copy()
        self.hull = np.ascontiguousarray(a["hull"] if a["hull"] is not None else np.zeros(n), np.uint8)
        self.row_ptr = np.ascontiguousarray(a["row_ptr"], np.int32)
        self.col = np.ascontiguousarray(a["col"], np.int32)
        self.c = np.ascontiguousarray(a["coupling"], np.float64).copy()
        types = a["types"]
        if a.get("geom") is not None:
            self.geom = np.ascontiguousarray(a["geom"], np.float64)
        else:
            eps = np.array([types[int(t)]["epsilon"] if int(t) in types else 1.0 for t in range(128)])
            ei = eps[np.repeat(self.type, np.diff(self.row_ptr))]
            ej = eps[self.type[self.col]]
            self.geom = self.c / (2 * ei * ej / (ei + ej))
        self.area_pos = np.ascontiguousarray(a["area_pos"] if a.get("area_pos") is not None else (self.geom != 0),
                                             np.uint8)
        self.phi = np.ascontiguousarray(a["phi"], np.float64).copy()
        self.volume = None if a.get("volume") is None else np.ascontiguousarray(a["volume"], np.float64)
        self.tet_v = None if a.get("tet_v") is None else np.ascontiguousarray(a["tet_v"], np.int32).reshape(-1)
        self.tet_n = None if a.get("tet_n") is None else np.ascontiguousarray(a["tet_n"], np.int32).reshape(-1)
        self.node_tet = a.get("node_tet")
        self.types = (orc_type * 128)()
        for tid, t in types.items():
            o = self.types[tid]
            o.present = 1
            o.removable = t["removable"]
            o.neumann = t["neumann"]
            o.dirichlet = t["dirichlet"]
            o.epsilon = t["epsilon"]
            o.evap_field = t["evap_field"]
            o.evap_energy = t["evap_energy"]
            o.charge_density = t["charge_density"]
            o.phi = t["phi"]
            o.mass = t["mass"]
            o.evap_charge = t["evap_charge"]
        self.q = np.zeros(n, np.float64)
        if self.volume is not None:
            rho = np.array([self.types[int(t)].charge_density for t in self.type])
            self.q = self.volume * rho / 8.85418781762e-12
        self.surface = np.zeros(n, np.uint8)
        self.top_z = float(self.xyz.reshape(-1, 3)[:, 2].max())
        self.m = orc_mesh(n, _p(self.xyz), _p(self.type), _p(self.hull), _p(self.row_ptr), _p(self.col), _p(self.c),
                          _p(self.geom), _p(self.area_pos), _p(self.phi), _p(self.q), _p(self.volume),
                          0 if self.tet_v is None else len(self.tet_v) // 4, _p(self.tet_v), _p(self.tet_n),
                          C.cast(self.types, C.c_void_p), _p(self.surface))
        self.L = lib()

    def residual(self) -> float:
        return self.L.orc_residual(C.byref(self.m))

    def solve(self, tol=1e-8, max_sweeps=1_000_000, omega=1.0):
        rel = C.c_double()
        s = self.L.orc_solve(C.byref(self.m), tol, max_sweeps, omega, C.byref(rel))
        return s, rel.value

    def relax(self, n: int) -> float:
        return self.L.orc_relax_cycles(C.byref(self.m), n)

    def local_set(self, node: int, shell: int) -> np.ndarray:
        """localRelax's cells (find_localNodes minus Dirichlet), ascending."""
        out = np.empty(self.m.n, np.int32)
        k = self.L.orc_local_set(C.byref(self.m), int(node), int(shell), _p(out), self.m.n)
        return out[:k].copy()

    def local_solve(self, cells: np.ndarray, tol: float = 1e-14, max_sweeps: int = 10_000_000) -> int:
        """The fixed point of localRelax on `cells`, the rest held."""
        c = np.ascontiguousarray(cells, np.int32)
        return self.L.orc_local_solve(C.byref(self.m), _p(c), len(c), tol, max_sweeps)


    def field_o1(self, node: int) -> np.ndarray:
        out = np.zeros(3, np.float64)
        self.L.orc_field_o1(C.byref(self.m), int(node), _p(out))
        return out

    def force(self, node: int) -> np.ndarray:
        out = np.zeros(3, np.float64)
        self.L.orc_force(C.byref(self.m), int(node), _p(out))
        return out

    def surface_init(self, vacuum_id: int) -> int:
        return self.L.orc_surface_init(C.byref(self.m), vacuum_id)

    def select(self):
        info = orc_select_info()
        ratio = np.zeros(self.n, np.float32)
        self.L.orc_select(C.byref(self.m), _p(ratio), C.byref(info))
        return info, ratio

    def select_mode(self, mode: int, temperature: float = 0.0):
        """(info, score) for probability mode 0..3 (surface_3d.cpp:220-399)."""
        info = orc_select_info()
        score = np.zeros(self.n, np.float32)
        self.L.orc_select_mode(C.byref(self.m), int(mode), float(temperature), _p(score), C.byref(info))
        return info, score

    def field_o2(self, i: int):
        E = np.zeros(3)
        q = C.c_double()
        ok = self.L.orc_field_o2(C.byref(self.m), int(i), _p(E), C.byref(q))
        return E, q.value, bool(ok)

    def pick(self, score: np.ndarray, total: float, u: float) -> int:
        return int(self.L.orc_pick(C.byref(self.m), _p(np.ascontiguousarray(score, np.float32)), float(total), float(u)))

    def take_away(self, node: int, vacuum_id: int) -> list[int]:
        det = np.zeros(512, np.int32)
        nd = self.L.orc_take_away(C.byref(self.m), int(node), vacuum_id, _p(det), 512)
        if nd < 0:
            raise RuntimeError(f"oracle: node {node} is not a surface cell")
        return det[:nd].tolist()

    def update_coordination(self):
        self.L.orc_update_coordination(C.byref(self.m))

    def trace(self, start, qm, tet_guess, dt0=1e-14, dt_min=1e-16, tol=1e-6, max_steps=200000,
              stepper_limit=1000) -> orc_impact:
        s = np.ascontiguousarray(start, np.float64)
        out = orc_impact()
        self.L.orc_trace(C.byref(self.m), _p(s), qm, int(tet_guess), dt0, dt_min, tol, max_steps, stepper_limit,
                         self.top_z, C.byref(out))
        return out

    def trace_ext(self, start, vel, qm, tet_guess, integrator=1, stepper=1, dt0=1e-14, dt_min=1e-16, tol=1e-6,
                  max_steps=200000, stepper_limit=1000) -> orc_impact:
        s = np.ascontiguousarray(start, np.float64)
        v = np.ascontiguousarray(vel, np.float64)
        out = orc_impact()
        self.L.orc_trace_ext(C.byref(self.m), _p(s), _p(v), qm, int(tet_guess), dt0, dt_min, tol, max_steps,
                             stepper_limit, self.top_z, int(integrator), int(stepper), C.byref(out))
        return out

    def trace_path(self, start, vel, qm, tet_guess, integrator=1, stepper=1, dt0=1e-14, dt_min=1e-16, tol=1e-6,
                   max_steps=200000, stepper_limit=1000, cap=100000):
        """(impact, points [k, 8]: time, position, velocity, tetrahedron;
        error estimate [6]) of one flight."""
        s = np.ascontiguousarray(start, np.float64)
        v = np.ascontiguousarray(vel, np.float64)
        out = orc_impact()
        path = np.zeros((cap, 8), np.float64)
        err = np.zeros(6, np.float64)
        self.L.orc_trace_path(C.byref(self.m), _p(s), _p(v), qm, int(tet_guess), dt0, dt_min, tol, max_steps,
                              stepper_limit, self.top_z, int(integrator), int(stepper), C.byref(out), cap, _p(path),
                              _p(err))
        n = 0 if out.status == -1 else min(out.steps + 2, cap)
        return out, path[:n], err

    def potential_at(self, p, tet_guess) -> float:
        s = np.ascontiguousarray(p, np.float64)
        return self.L.orc_potential_at(C.byref(self.m), _p(s), int(tet_guess))


def stagnated(deviations, queue: int, cycle: int) -> bool:
    """The RelaxationFault rule of relax(thr, cycle, queue) on a deviation history."""
    d = np.ascontiguousarray(deviations, np.float64)
    return bool(lib().orc_stagnated(_p(d), len(d), int(queue), int(cycle)))
