"""Python mirror of the reference's split-solver / simulator interface.

Names, argument meaning and error behaviour follow the reference:

* ``SplitSolver.solve(in, out, dtdh)`` -- solver::SplitSolver::solve
  (solver/split_solver.hpp:105-115): all sweeps x, y, z with the reference's
  buffer swap; returns the (in, out) pair after the swap, out holding the
  new state.
* ``SimulatorImpl`` -- sim::SimulatorImpl (simulator/simulator_impl.hpp:43-512):
  configure_resolution / configure_dimension / configure_sim_time /
  configure_cfl / configure_max_iterations, fill_data, simulate,
  write_results.

Device memory comes from torch (plumbing only); every numerical operation is a
call into libfluidity_b200.so through the C ABI.  Errors raise
``capi.FlError`` instead of terminating the process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import capi

_DT = {"f64": torch.float64, "f32": torch.float32}


def _stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def state_tensor(shape, dtype: str = "f64", device="cuda", pitch: int | None = None):
    """Empty SoA state buffer: (dims + 2, pitch) with pitch >= prod(shape)."""
    cells = int(np.prod(shape))
    pitch = cells if pitch is None else pitch
    return torch.empty((len(shape) + 2, pitch), dtype=_DT[dtype], device=device)


class SplitSolver:
    """Dimensionally split MUSCL-Hancock / HLLC|FORCE step on one GPU.

    p_inf = 0 is the ideal gas (material/ideal_gas.hpp); p_inf > 0 the
    stiffened fluid StiffFluid(gamma, p_inf) (material/stiff_fluid.hpp:38-133),
    through the C ABI's fl_material entry points.

    workspace=True (the default) sweeps through fl_split_sweep_ws /
    fl_split_solve_ws with a workspace allocated once here: strips taken
    dynamically and, in 3-D, the register walk.  workspace=False takes the
    plain entry points (one strip per warp; 3-D through the tile kernel)."""

    def __init__(self, shape, dtype: str = "f64", flux: str = "hllc",
                 limiter: str = "vanleer", recon: str = "muscl", gamma: float = 1.4,
                 boundary_mask: int = 0, flatten: bool = True, pitch: int | None = None,
                 p_inf: float = 0.0, workspace: bool = True):
        self.shape = tuple(int(v) for v in shape)
        self.dims = len(self.shape)
        self.dtype = dtype
        self.gamma = float(gamma)
        self.p_inf = float(p_inf)
        self.material = capi.Material(self.gamma, self.p_inf)
        self.boundary_mask = int(boundary_mask)
        self.policy = capi.policy_bits(dtype, flux, limiter, recon, flatten)
        self.grid = capi.Grid.make(self.shape, pitch)
        self.lib = capi.load()
        self.workspace = None
        if workspace:
            nbytes = self.lib.fl_workspace_bytes(C.byref(self.grid), self.policy)
            if nbytes < 0:
                capi.check(capi.FL_EINVAL, self.lib)
            self.workspace = torch.zeros(int(nbytes), dtype=torch.uint8, device="cuda")

    def _ws(self):
        return C.c_void_p(self.workspace.data_ptr())

    def workspace_status(self, stream=None) -> int:
        """The workspace's status word (0, or FL_ETIMEOUT); synchronises."""
        st = C.c_int()
        capi.check(self.lib.fl_workspace_status(self._ws(), _stream_ptr(stream), C.byref(st)),
                   self.lib)
        return st.value

    def new_state(self):
        return state_tensor(self.shape, self.dtype, pitch=self.grid.pitch)

    def sweep(self, src, dst, dim: int, dtdh: float, max_ws=None, stream=None):
        """One dimensional sweep; max_ws (1-element float64 cuda tensor) receives
        the max wavespeed of dst."""
        ws = None if max_ws is None else C.c_void_p(max_ws.data_ptr())
        args = (C.c_void_p(src.data_ptr()), C.c_void_p(dst.data_ptr()))
        if self.workspace is not None:
            rc = self.lib.fl_split_sweep_ws(C.byref(self.grid), int(dim), *args,
                                            C.byref(self.material), float(dtdh), self.policy,
                                            self.boundary_mask, ws, self._ws(), _stream_ptr(stream))
        elif self.p_inf != 0.0:
            rc = self.lib.fl_split_sweep_mat(C.byref(self.grid), int(dim), *args,
                                             C.byref(self.material), float(dtdh), self.policy,
                                             self.boundary_mask, ws, _stream_ptr(stream))
        else:
            rc = self.lib.fl_split_sweep(C.byref(self.grid), int(dim), *args, self.gamma,
                                         float(dtdh), self.policy, self.boundary_mask, ws,
                                         _stream_ptr(stream))
        capi.check(rc, self.lib)

    def solve(self, src, dst, dtdh: float, max_ws=None, stream=None):
        """All sweeps; returns (in, out) after the reference's swap."""
        pin = C.c_void_p(src.data_ptr())
        pout = C.c_void_p(dst.data_ptr())
        ws = None if max_ws is None else C.c_void_p(max_ws.data_ptr())
        if self.workspace is not None:
            rc = self.lib.fl_split_solve_ws(C.byref(self.grid), C.byref(pin), C.byref(pout),
                                            C.byref(self.material), float(dtdh), self.policy,
                                            self.boundary_mask, ws, self._ws(), _stream_ptr(stream))
        elif self.p_inf != 0.0:
            rc = self.lib.fl_split_solve_mat(C.byref(self.grid), C.byref(pin), C.byref(pout),
                                             C.byref(self.material), float(dtdh), self.policy,
                                             self.boundary_mask, ws, _stream_ptr(stream))
        else:
            rc = self.lib.fl_split_solve(C.byref(self.grid), C.byref(pin), C.byref(pout),
                                         self.gamma, float(dtdh), self.policy,
                                         self.boundary_mask, ws, _stream_ptr(stream))
        capi.check(rc, self.lib)
        by_ptr = {src.data_ptr(): src, dst.data_ptr(): dst}
        return by_ptr[pin.value], by_ptr[pout.value]

    def max_wavespeed(self, state, stream=None) -> torch.Tensor:
        out = torch.empty(1, dtype=torch.float64, device=state.device)
        if self.p_inf != 0.0:
            rc = self.lib.fl_max_wavespeed_mat(C.byref(self.grid), C.c_void_p(state.data_ptr()),
                                               C.byref(self.material), self.policy,
                                               C.c_void_p(out.data_ptr()), _stream_ptr(stream))
        else:
            rc = self.lib.fl_max_wavespeed(C.byref(self.grid), C.c_void_p(state.data_ptr()),
                                           self.gamma, self.policy, C.c_void_p(out.data_ptr()),
                                           _stream_ptr(stream))
        capi.check(rc, self.lib)
        return out

    def fill_riemann(self, states_prim, out=None, stream=None):
        """Orthant initial data from 2**dims primitive states (rho, p, v...)."""
        sp = np.ascontiguousarray(states_prim, dtype=np.float64).reshape(2 ** self.dims,
                                                                          self.dims + 2)
        out = self.new_state() if out is None else out
        if self.p_inf != 0.0:
            rc = self.lib.fl_fill_riemann_mat(C.byref(self.grid), sp.ctypes.data_as(C.c_void_p),
                                              C.byref(self.material), self.policy,
                                              C.c_void_p(out.data_ptr()), _stream_ptr(stream))
        else:
            rc = self.lib.fl_fill_riemann(C.byref(self.grid), sp.ctypes.data_as(C.c_void_p),
                                          self.gamma, self.policy, C.c_void_p(out.data_ptr()),
                                          _stream_ptr(stream))
        capi.check(rc, self.lib)
        return out


class Simulation:
    """Device-resident time loop (fl_sim_*): SimulatorImpl::simulate."""

    def __init__(self, solver: SplitSolver):
        self.solver = solver
        self.lib = solver.lib
        h = C.c_void_p()
        capi.check(self.lib.fl_sim_create(C.byref(h), C.byref(solver.grid), solver.gamma,
                                          solver.policy, solver.boundary_mask), self.lib)
        self.handle = h
        if solver.p_inf != 0.0:
            capi.check(self.lib.fl_sim_set_material(h, C.byref(solver.material)), self.lib)
        self._bufs = {}

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.fl_sim_destroy(h)
            except Exception:
                pass
            self.handle = None

    def begin(self, a, b, cfl, res, sim_time, max_iters, stream=None):
        self._bufs = {a.data_ptr(): a, b.data_ptr(): b}
        capi.check(self.lib.fl_sim_begin(self.handle, C.c_void_p(a.data_ptr()),
                                         C.c_void_p(b.data_ptr()), float(cfl), float(res),
                                         float(sim_time), int(max_iters), _stream_ptr(stream)),
                   self.lib)

    def steps(self, n, stream=None):
        capi.check(self.lib.fl_sim_steps(self.handle, int(n), _stream_ptr(stream)), self.lib)

    def status(self, stream=None, allow_nan=False):
        """(iters, run_time, done, result buffer); a non-finite wavespeed raises
        FlError(FL_ENAN) unless allow_nan, which reports the steps completed."""
        it = C.c_int64()
        rt = C.c_double()
        done = C.c_int()
        res = C.c_void_p()
        rc = self.lib.fl_sim_status(self.handle, _stream_ptr(stream), C.byref(it), C.byref(rt),
                                    C.byref(done), C.byref(res))
        if not (allow_nan and rc == capi.FL_ENAN):
            capi.check(rc, self.lib)
        return int(it.value), float(rt.value), bool(done.value), self._bufs[res.value]

    def run(self, a, b, cfl, res, sim_time, max_iters, stream=None):
        """begin + steps until done; returns (result, iters, run_time)."""
        self._bufs = {a.data_ptr(): a, b.data_ptr(): b}
        it = C.c_int64()
        rt = C.c_double()
        out = C.c_void_p()
        capi.check(self.lib.fl_simulate(self.handle, C.c_void_p(a.data_ptr()),
                                        C.c_void_p(b.data_ptr()), float(cfl), float(res),
                                        float(sim_time), int(max_iters), _stream_ptr(stream),
                                        C.byref(it), C.byref(rt), C.byref(out)), self.lib)
        return self._bufs[out.value], int(it.value), float(rt.value)


class HostPipeline:
    """Whole simulations from host memory to host memory (fl_host_pipe_*):
    job k + 1's upload and job k - 1's download overlap job k's compute.
    Host tensors should be pinned (``torch.empty(..., pin_memory=True)``) and
    shaped like ``solver.new_state()``."""

    def __init__(self, solver: SplitSolver, sets: int = 3):
        self.solver = solver
        self.lib = solver.lib
        h = C.c_void_p()
        capi.check(self.lib.fl_host_pipe_create(C.byref(h), C.byref(solver.grid), solver.gamma,
                                                solver.policy, solver.boundary_mask, int(sets)),
                   self.lib)
        self.handle = h
        if solver.p_inf != 0.0:
            capi.check(self.lib.fl_host_pipe_set_material(h, C.byref(solver.material)),
                       self.lib)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.fl_host_pipe_destroy(h)
            except Exception:
                pass
            self.handle = None

    def run(self, host_in, host_out, cfl, res, sim_time, max_iters):
        """host_in / host_out: equal-length lists of pinned host tensors.
        Returns [(iters, run_time)] per job."""
        n = len(host_in)
        if len(host_out) != n:
            raise ValueError("host_in and host_out differ in length")
        ins = (C.c_void_p * n)(*[t.data_ptr() for t in host_in])
        outs = (C.c_void_p * n)(*[t.data_ptr() for t in host_out])
        for t in list(host_in) + list(host_out):
            if t.is_cuda or t.numel() * t.element_size() < self.lib.fl_state_bytes(
                    C.byref(self.solver.grid), self.solver.policy):
                raise ValueError("host buffers must be host tensors of a whole state")
        its = (C.c_int64 * max(n, 1))()
        rts = (C.c_double * max(n, 1))()
        capi.check(self.lib.fl_host_pipe_run(self.handle, n, ins, outs, float(cfl), float(res),
                                             float(sim_time), int(max_iters), its, rts),
                   self.lib)
        return [(int(its[k]), float(rts[k])) for k in range(n)]


def write_separate_raw(u, shape, gamma, prefix, sim_time):
    """write_results_separate_raw (simulator/simulator_impl.hpp:360-420) for a
    host state u ((dims + 2, >= cells) conservative planes): one file per
    primitive variable, <prefix>_<name>_<sim_time>.dat, values formatted as a
    C++ stream's default (%g) each followed by a space; 1-D: one line then a
    blank line; 2-D: one line per row; 3-D: the 2-D files of plane z under
    <prefix>_<z>.  Primitives are computed in the state's precision."""
    u = np.asarray(u)
    D = len(shape)
    cells = int(np.prod(shape))
    T = u.dtype.type
    rho = u[0, :cells]
    v = [u[2 + d, :cells] / rho for d in range(D)]
    v2 = T(0)
    for d in range(D):
        v2 = v2 + v[d] * v[d]
    p = (T(gamma) - T(1)) * (u[1, :cells] - T(0.5) * rho * v2)
    prim = [rho, p] + v
    names = ["rho", "p", "v_x", "v_y", "v_z"][:D + 2]
    nx = shape[0]
    ny = shape[1] if D >= 2 else 1
    nz = shape[2] if D == 3 else 1
    stamp = f"{float(sim_time):f}"
    paths = []
    for z in range(nz):
        pre = f"{prefix}_{z}" if D == 3 else prefix
        for k, name in enumerate(names):
            path = f"{pre}_{name}_{stamp}.dat"
            plane = prim[k].reshape(nz, ny, nx)[z]
            with open(path, "w") as f:
                for y in range(ny):
                    f.write("".join("%g " % float(val) for val in plane[y]) + "\n")
                if D == 1:
                    f.write("\n")
            paths.append(path)
    return paths


class SimulatorImpl:
    """sim::SimulatorImpl (simulator/simulator_impl.hpp:43-512) on one B200.

    Defaults follow SimTraits (simulator/simulator_traits.hpp:44-58) except the
    limiter and flux, which the caller picks (the reference's
    ``create_default`` uses Superbee + FORCE)."""

    def __init__(self, dims: int = 1, dtype: str = "f64", flux: str = "force",
                 limiter: str = "superbee", recon: str = "muscl", gamma: float = 1.4,
                 boundary_mask: int = 0, p_inf: float = 0.0):
        self.dims = dims
        self.kw = dict(dtype=dtype, flux=flux, limiter=limiter, recon=recon, gamma=gamma,
                       boundary_mask=boundary_mask, p_inf=p_inf)
        self.res = 0.0
        self.extent = [(0.0, 1.0)] * dims
        self.sim_time = 0.0
        self.cfl = 0.9
        self.max_iters = (1 << 63) - 1
        self.state = None
        self.iters = 0
        self.run_time = 0.0

    # simulator_impl.hpp:260-291
    def configure_resolution(self, res: float):
        self.res = float(res)

    def configure_dimension(self, dim: int, start: float, end: float):
        self.extent[dim] = (float(start), float(end))

    def configure_sim_time(self, t: float):
        self.sim_time = float(t)

    def configure_cfl(self, cfl: float):
        self.cfl = float(cfl)

    def configure_max_iterations(self, n: int):
        self.max_iters = int(n)

    def shape(self):
        # Domain::elements (simulator/domain.hpp:69-73): size_t((end - start) / res)
        return tuple(int((e - s) / self.res) for s, e in self.extent)

    def fill_data(self, states_prim):
        """Orthant initial data; states_prim is (2**dims, dims + 2) primitive."""
        self.solver = SplitSolver(self.shape(), **self.kw)
        self.state = self.solver.fill_riemann(states_prim)

    def simulate(self):
        if self.state is None:
            raise RuntimeError("fill_data must be called before simulate")
        sim = Simulation(self.solver)
        other = self.solver.new_state()
        self.state, self.iters, self.run_time = sim.run(self.state, other, self.cfl, self.res,
                                                        self.sim_time, self.max_iters)
        torch.cuda.synchronize()
        del sim

    def states(self) -> np.ndarray:
        return self.state.double().cpu().numpy()

    def write_results_separate_raw(self, prefix: str):
        """One file per primitive variable (simulator_impl.hpp:413-420)."""
        return write_separate_raw(self.states(), self.shape(), self.kw["gamma"], prefix,
                                  self.sim_time)

    @classmethod
    def from_settings(cls, text: str, gamma: float = 1.4, boundary_mask: int = 0):
        """A simulator configured by a fluidity settings text's
        "simulator : { ... }" block (setting/simulator_parameter.hpp), the
        run-time form of OptionManager::create (setting/option_manager.hpp
        :241-246)."""
        pol, dims = capi.policy_from_settings(text)
        sim = cls(dims=dims, gamma=gamma, boundary_mask=boundary_mask)
        sim.kw["dtype"] = "f32" if pol & 1 else "f64"
        sim.kw["flux"] = {0: "hllc", 1: "force", 2: "lf", 3: "richtmyer"}[(pol >> 1) & 3]
        sim.kw["limiter"] = "superbee" if (pol >> 3) & 1 else "vanleer"
        sim.kw["recon"] = "basic" if (pol >> 4) & 1 else "muscl"
        return sim

    def write_results(self, prefix: str):
        """ASCII columns: position(s) then rho, p, v... (primitive), one cell per
        line, in the spirit of SimulatorImpl::write_results
        (simulator/simulator_impl.hpp:350-358,436-508)."""
        u = self.states()[:, : int(np.prod(self.shape()))]
        D = self.dims
        g = self.kw["gamma"]
        rho = u[0]
        v = u[2:2 + D] / rho
        p = (g - 1.0) * (u[1] - 0.5 * rho * np.sum(v * v, axis=0))
        shape = self.shape()
        idx = np.indices(shape[::-1]).reshape(D, -1)[::-1]
        pos = [(idx[d] + 0.5) * self.res + self.extent[d][0] for d in range(D)]
        cols = np.vstack(pos + [rho, p] + [v[d] for d in range(D)]).T
        names = ["x", "y", "z"][:D] + ["rho", "p"] + ["v_" + c for c in "xyz"[:D]]
        np.savetxt(prefix + ".dat", cols, header=" ".join(names))
