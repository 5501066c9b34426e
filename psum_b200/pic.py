"""Python mirror of the particle-kernel set (include/psum_pic.h).

``ParticleContext`` owns one ``psum_pic_ctx``: a grid (``simple_grid<D>``
conventions), one or more species, and the device state.  It plays the role
of PSuM's ``particle_group`` + ``device_field`` pair for the electrostatic
step (src/particle_container/particle_group.hpp, src/field/device_field.hpp):
load particles, push with the CIC gather, deposit, sort/bin by cell, and run
whole steps through a solver handle.
"""
import ctypes as C

import numpy as np

from ._lib import GridDesc, SpeciesDesc, check, lib
from .field_solver import _ptr, _ready, _stream_handle

MIXED, FP64 = 0, 1
LEAPFROG, BORIS = 0, 1


class ParticleContext:
    def __init__(self, cells, lower, upper, periodic, precision=MIXED):
        g = GridDesc()
        g.dim = len(cells)
        for a in range(3):
            g.cells[a] = int(cells[a]) if a < g.dim else 1
            g.lower[a] = float(lower[a]) if a < g.dim else 0.0
            g.upper[a] = float(upper[a]) if a < g.dim else 1.0
            g.periodic[a] = int(bool(periodic[a])) if a < g.dim else 0
        self.desc = g
        self.dim = g.dim
        self.cells = list(cells)
        self.precision = precision
        self.n_nodes = int(np.prod([c + 1 for c in cells]))
        self.species = []
        h = C.c_void_p()
        check(lib().psum_pic_create(C.byref(g), precision, C.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            check(lib().psum_pic_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream):
        """Run later work on `stream` (torch stream or handle); None = own stream.
        With the caller's stream set, torch work and library work are ordered
        by that stream and no extra synchronisation is needed."""
        self._stream = stream
        check(lib().psum_pic_set_stream(self.handle, _stream_handle(stream)))

    def _order(self, *tensors):
        if getattr(self, "_stream", None) is None:
            _ready(*tensors)

    def set_options(self, options):
        check(lib().psum_pic_set_options(self.handle, options.encode()))

    def add_species(self, charge, mass, weight, capacity):
        d = SpeciesDesc(float(charge), float(mass), float(weight))
        sid = C.c_int()
        check(lib().psum_pic_add_species(self.handle, C.byref(d), int(capacity), C.byref(sid)))
        self.species.append((charge, mass, weight))
        return sid.value

    def load(self, species, pos, vel):
        """pos: (dim, n) float64, vel: (3, n) float64 host arrays (numpy) or
        device tensors (torch, float64, contiguous)."""
        if hasattr(pos, "data_ptr") and getattr(pos, "is_cuda", False):
            n = pos.shape[1]
            _ready(pos, vel)
            check(lib().psum_pic_load_device(self.handle, species, n, pos.data_ptr(), vel.data_ptr()))
        else:
            pos = np.ascontiguousarray(pos, np.float64)
            vel = np.ascontiguousarray(vel, np.float64)
            n = pos.shape[1]
            check(lib().psum_pic_load(self.handle, species, n, _ptr(pos), _ptr(vel)))

    def append(self, species, pos, vel):
        """Add particles after the stored ones (PSuM's particle_group::insert);
        the same array conventions as load.  The species is unsorted afterwards
        and, as after load, deposit() must run before the next step."""
        if hasattr(pos, "data_ptr") and getattr(pos, "is_cuda", False):
            n = pos.shape[1]
            _ready(pos, vel)
            check(lib().psum_pic_append_device(self.handle, species, n, pos.data_ptr(), vel.data_ptr()))
        else:
            pos = np.ascontiguousarray(pos, np.float64)
            vel = np.ascontiguousarray(vel, np.float64)
            n = pos.shape[1]
            check(lib().psum_pic_append(self.handle, species, n, _ptr(pos), _ptr(vel)))

    def count(self, species):
        ns, nv = C.c_ulonglong(), C.c_ulonglong()
        check(lib().psum_pic_count(self.handle, species, C.byref(ns), C.byref(nv)))
        return ns.value, nv.value

    def get_state(self, species):
        ns, _ = self.count(species)
        pos = np.zeros((self.dim, ns))
        vel = np.zeros((3, ns))
        check(lib().psum_pic_get_state(self.handle, species, _ptr(pos), _ptr(vel)))
        return pos, vel

    def get_state_device(self, species):
        """The stored particles as (dim, n) and (3, n) float64 CUDA tensors
        (invalid particles have x = NaN): the positions the B-spline
        functions of psum_b200.interp take."""
        import torch
        ns, _ = self.count(species)
        pos = torch.empty((self.dim, ns), dtype=torch.float64, device="cuda")
        vel = torch.empty((3, ns), dtype=torch.float64, device="cuda")
        self._order(pos, vel)
        check(lib().psum_pic_get_state_device(self.handle, species, _ptr(pos), _ptr(vel)))
        return pos, vel

    def get_keys(self, species, out):
        self._order(out)
        check(lib().psum_pic_get_keys(self.handle, species, _ptr(out)))

    def sort(self):
        check(lib().psum_pic_sort(self.handle))

    def bin(self, species, keys, counts, offsets, perm):
        n = C.c_ulonglong()
        self._order(keys, counts, offsets, perm)
        check(lib().psum_pic_bin(self.handle, species, _ptr(keys), _ptr(counts), _ptr(offsets), _ptr(perm),
                                 C.byref(n)))
        return n.value

    def deposit(self):
        check(lib().psum_pic_deposit(self.handle))

    def rho(self, background, out):
        self._order(out)
        check(lib().psum_pic_rho(self.handle, float(background), _ptr(out)))

    def density(self, species, out):
        self._order(out)
        check(lib().psum_pic_density(self.handle, species, _ptr(out)))

    def push(self, phi, dt, pusher=LEAPFROG, B=(0.0, 0.0, 0.0)):
        Bv = (C.c_double * 3)(*B)
        self._order(phi)
        check(lib().psum_pic_push(self.handle, _ptr(phi), float(dt), pusher, Bv))

    def losses(self, reset=True):
        out = np.zeros(len(self.species) * 2 * self.dim, np.uint64)
        check(lib().psum_pic_get_losses(self.handle, _ptr(out), int(reset)))
        return out.reshape(len(self.species), self.dim, 2)

    def join(self):
        """Order the context's stream after the last step's deferred second
        pass (see psum_pic_join); the state readers do this themselves."""
        check(lib().psum_pic_join(self.handle))

    def step(self, solver, background, rho, phi, dt, pusher=LEAPFROG, B=(0.0, 0.0, 0.0)):
        Bv = (C.c_double * 3)(*B)
        self._order(rho, phi)
        check(lib().psum_pic_step(self.handle, solver.handle, float(background), _ptr(rho), _ptr(phi), float(dt),
                                  pusher, Bv))

    def set_timing(self, enable=True):
        check(lib().psum_pic_set_timing(self.handle, int(bool(enable))))

    def get_timing(self, reset=True):
        """Accumulated ms and counts per step phase: rho, solve, push, sort, diag (the reduction of the
        per-step diagnostics of option 'diagnostics 1')."""
        names = ("rho", "solve", "push", "sort", "diag")
        ms = np.zeros(len(names))
        cnt = np.zeros(len(names), np.int32)
        check(lib().psum_pic_get_phase_times(self.handle, _ptr(ms), _ptr(cnt), len(names), int(reset)))
        return dict(zip(names, zip(ms.tolist(), cnt.tolist())))

    def diagnostics(self, phi, epsilon):
        out = np.zeros(len(self.species) + 2)
        self._order(phi)
        check(lib().psum_pic_diagnostics(self.handle, _ptr(phi), float(epsilon), _ptr(out)))
        return {"kinetic": out[:len(self.species)].copy(), "field": out[-2], "charge": out[-1]}

    def step_diagnostics(self, epsilon):
        """The diagnostics the last psum_pic_step computed (option 'diagnostics 1'): kinetic energy per
        species after the push, field energy of the step's phi, charge of the step's density."""
        out = np.zeros(len(self.species) + 2)
        check(lib().psum_pic_get_step_diagnostics(self.handle, float(epsilon), _ptr(out)))
        return {"kinetic": out[:len(self.species)].copy(), "field": out[-2], "charge": out[-1]}

    def device_errors(self):
        f = C.c_uint()
        check(lib().psum_pic_device_errors(self.handle, C.byref(f)))
        return f.value

    # ---- differentiable runs: state snapshots and the adjoint of one step
    def state_bytes(self, species):
        b = C.c_ulonglong()
        check(lib().psum_pic_state_bytes(self.handle, species, C.byref(b)))
        return b.value

    def save_state(self, species, dst):
        """Copy the species' state into the device uint8 tensor `dst`."""
        self._order(dst)
        check(lib().psum_pic_save_state(self.handle, species, _ptr(dst)))

    def restore_state(self, species, src):
        self._order(src)
        check(lib().psum_pic_restore_state(self.handle, species, _ptr(src)))

    def adjoint_push(self, species, phi, dt, lam_x, lam_v, mu):
        """Adjoint of the leapfrog kick and move at the current state: lam_x
        (dim, n) and lam_v (3, n) go from the adjoints of the new state to
        those of the old state (float32 in MIXED contexts, float64 in FP64);
        the adjoint of phi is added to mu (float64 per node)."""
        self._order(phi, lam_x, lam_v, mu)
        check(lib().psum_pic_adjoint_push(self.handle, species, _ptr(phi), float(dt), _ptr(lam_x), _ptr(lam_v),
                                          _ptr(mu)))

    def adjoint_deposit(self, species, nu, lam_x):
        """lam_x += gather of the CIC gradient of nu = dL/drho (float64 per node)."""
        self._order(nu, lam_x)
        check(lib().psum_pic_adjoint_deposit(self.handle, species, _ptr(nu), _ptr(lam_x)))

