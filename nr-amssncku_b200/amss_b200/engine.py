"""Batched, device-resident evolution engine (amss_engine_* of include/amss_b200.h).

The engine plays the role of the reference's level step (bssn_class::Step,
bssn_class.C:2981-3915): it owns every block's state in HBM and advances all
blocks of a level by one RK4 step with four kernel launches.
"""
import ctypes

import numpy as np

from ._lib import _DP, _IP, AmssError, check, last_error, lib


class _Params(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("symmetry", ctypes.c_int),
                ("eps", ctypes.c_double), ("chitiny", ctypes.c_double), ("kernel", ctypes.c_int),
                ("formulation", ctypes.c_int)]


class Engine:
    """One hierarchy of blocks on the current CUDA device.

    precision: "fp64" or "mixed" (FP32 stencils and stages, FP64 state,
    accumulator and update).  kernel: "split" (a stencil pass through shared
    memory, then the pointwise RHS and RK4 update) or "fused" (one pass,
    every stencil from global memory).  chitiny is BSSN::chitiny as the par file gives
    it (1e-5); the engine shifts it by -1 as bssn_class.C:179 does.
    formulation: "bssn" (24 fields) or "z4c" (25 fields, Theta last; split
    kernel only)."""

    _create = "amss_engine_create"

    def __init__(self, precision="fp64", symmetry=0, eps=0.1, chitiny=1e-5, kernel="split", formulation="bssn"):
        if formulation not in ("bssn", "z4c"):
            raise AmssError("formulation must be 'bssn' or 'z4c'")
        self.nf = 25 if formulation == "z4c" else 24
        self.params = dict(precision=precision, symmetry=symmetry, eps=eps, chitiny=chitiny, kernel=kernel,
                           formulation=formulation)
        prm = _Params(1 if precision == "mixed" else 0, symmetry, eps, chitiny - 1.0, 0 if kernel == "split" else 1,
                      1 if formulation == "z4c" else 0)
        self._h = getattr(lib(), self._create)(ctypes.byref(prm))
        if not self._h:
            raise AmssError(f"{self._create} failed: " + last_error())
        self.blocks = []
        self._ntrack = 0
        self.rank, self.nranks = 0, 1

    def close(self):
        if self._h:
            lib().amss_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_block(self, level, ex, bbox, patch_bbox):
        exa = (ctypes.c_int * 3)(*ex)
        bb = (ctypes.c_double * 6)(*bbox)
        pb = (ctypes.c_double * 6)(*patch_bbox)
        bid = check(lib().amss_engine_add_block(self._h, level, exa, bb, pb), "amss_engine_add_block")
        self.blocks.append(tuple(ex))
        return bid

    def set_grid(self, x0, h0):
        check(lib().amss_engine_set_grid(self._h, (ctypes.c_double * 3)(*x0), h0), "amss_engine_set_grid")

    def add_amr_block(self, level, patch, org, ex, own_lo, own_hi, phys_lo, phys_hi, buffer):
        I3 = ctypes.c_int * 3
        bid = check(lib().amss_engine_add_amr_block(self._h, level, patch, I3(*org), I3(*ex), I3(*own_lo), I3(*own_hi),
                                                    I3(*phys_lo), I3(*phys_hi), buffer), "amss_engine_add_amr_block")
        self.blocks.append(tuple(ex))
        return bid

    @classmethod
    def from_hierarchy(cls, H, rank=0, nranks=1, owners=None, **kw):
        """An engine over every block of an amss_b200.hierarchy.Hierarchy,
        block ids equal to their index in H.blocks.  With nranks > 1 it is
        rank `rank` of a job whose block owners are `owners` (one rank per
        block, amss_b200.dist.partition): it holds and steps only its own."""
        e = cls(**kw)
        e.set_grid((H.x0,) * 3, H.h0)
        for lev, patches in enumerate(H.levels):
            for pid, p in enumerate(patches):
                for bi in p.blocks:
                    b = H.blocks[bi]
                    got = e.add_amr_block(lev, pid, b.org, b.ex, b.own_lo, b.own_hi, p.lo, p.hi, p.buffer)
                    assert got == bi
        if nranks > 1 or rank:
            e.set_rank(rank, nranks)
            if owners is None or len(owners) != len(H.blocks):
                raise AmssError("from_hierarchy: nranks > 1 needs one owner per block")
            for bi, o in enumerate(owners):
                e.set_block_owner(bi, int(o))
        e.commit()
        return e

    def set_rank(self, rank, nranks):
        """This engine is rank `rank` of `nranks` (before commit)."""
        check(lib().amss_engine_set_rank(self._h, int(rank), int(nranks)), "amss_engine_set_rank")
        self.rank, self.nranks = int(rank), int(nranks)

    def set_block_owner(self, block, owner):
        check(lib().amss_engine_set_block_owner(self._h, int(block), int(owner)), "amss_engine_set_block_owner")

    def coarse_step(self, dt0):
        check(lib().amss_engine_coarse_step(self._h, dt0), "amss_engine_coarse_step")

    def run_coarse_graph(self, dt0, nsteps, replays=1):
        check(lib().amss_engine_run_coarse_graph(self._h, dt0, nsteps, replays), "amss_engine_run_coarse_graph")

    def level_points(self, level):
        return lib().amss_engine_level_points(self._h, level)

    def commit(self):
        check(lib().amss_engine_commit(self._h), "amss_engine_commit")

    def set_state(self, block, state):
        state = np.ascontiguousarray(state, dtype=np.float64)
        ex = self.blocks[block]
        if state.shape != (self.nf, ex[2], ex[1], ex[0]):
            raise AmssError(f"set_state: state must have shape {(self.nf, ex[2], ex[1], ex[0])}, got {state.shape}")
        check(lib().amss_engine_set_state(self._h, block, state.ctypes.data_as(_DP)), "amss_engine_set_state")

    def get_state(self, block, out=None):
        ex = self.blocks[block]
        if out is None:
            out = np.empty((self.nf, ex[2], ex[1], ex[0]))
        if out.dtype != np.float64 or not out.flags.c_contiguous or out.shape != (self.nf, ex[2], ex[1], ex[0]):
            raise AmssError(f"get_state: out must be a C-contiguous float64 ({self.nf}, ez, ey, ex) array")
        check(lib().amss_engine_get_state(self._h, block, out.ctypes.data_as(_DP)), "amss_engine_get_state")
        return out

    def set_time_level(self, block, back, state):
        """A block's state `back` level steps before the current one (0..2)."""
        state = np.ascontiguousarray(state, dtype=np.float64)
        ex = self.blocks[block]
        if state.shape != (self.nf, ex[2], ex[1], ex[0]):
            raise AmssError(f"set_time_level: state must have shape {(self.nf, ex[2], ex[1], ex[0])}")
        check(lib().amss_engine_set_time_level(self._h, block, back, state.ctypes.data_as(_DP)),
              "amss_engine_set_time_level")

    def get_time_level(self, block, back):
        ex = self.blocks[block]
        out = np.empty((self.nf, ex[2], ex[1], ex[0]))
        check(lib().amss_engine_get_time_level(self._h, block, back, out.ctypes.data_as(_DP)),
              "amss_engine_get_time_level")
        return out

    def level_steps(self, level):
        n = ctypes.c_int()
        check(lib().amss_engine_level_clock(self._h, level, ctypes.byref(n)), "amss_engine_level_clock")
        return n.value

    def set_level_steps(self, level, steps):
        check(lib().amss_engine_set_level_clock(self._h, level, int(steps)), "amss_engine_set_level_clock")

    def state_device(self, block):
        ptr = ctypes.c_void_p()
        fs = ctypes.c_longlong()
        check(lib().amss_engine_state_device(self._h, block, ctypes.byref(ptr), ctypes.byref(fs)),
              "amss_engine_state_device")
        return ptr.value, fs.value

    def enforce(self):
        check(lib().amss_engine_enforce(self._h), "amss_engine_enforce")

    def step(self, level, dt):
        check(lib().amss_engine_step_level(self._h, level, dt), "amss_engine_step_level")

    def regrid_fill(self, old, level, back):
        """Fill `level`, time level `back` (0 current, 1 previous), from the
        engine this one replaces (amss_engine_regrid_fill)."""
        check(lib().amss_engine_regrid_fill(self._h, old._h, level, back), "amss_engine_regrid_fill")

    def set_level_tiling(self, level, tile_w=0, zsplit=1):
        """Stencil-pass tiling of one level (amss_engine_set_level_tiling):
        tile width 8..64 (0: default) and z-slabs per block."""
        check(lib().amss_engine_set_level_tiling(self._h, level, int(tile_w), int(zsplit)),
              "amss_engine_set_level_tiling")

    def set_level_occupancy(self, level, occ):
        """Compiled form of a level's stencil pass: 0 (two resident CTAs per
        SM) or 1 (four in FP64, three in FP32)."""
        check(lib().amss_engine_set_level_occupancy(self._h, level, int(occ)), "amss_engine_set_level_occupancy")

    def level_occupancy(self, level):
        o = ctypes.c_int()
        check(lib().amss_engine_get_level_occupancy(self._h, level, ctypes.byref(o)), "amss_engine_get_level_occupancy")
        return o.value

    def final_region(self, level):
        """(pad, points) of a level's final substep in a coarse step: pad 2,
        the owned cells within 2 of the physical box (the rest are overwritten
        by the prolongation unread); -1, no such regions (the owned cells, where
        the sync fills every ghost, else whole arrays).  points: the cells it
        updates on this engine's blocks."""
        pad, pts = ctypes.c_int(), ctypes.c_longlong()
        check(lib().amss_engine_level_final_region(self._h, level, ctypes.byref(pad), ctypes.byref(pts)),
              "amss_engine_level_final_region")
        return pad.value, pts.value

    def level_tiling(self, level):
        """(tile width as set, z-slabs, stencil work items) of one level."""
        w, z, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().amss_engine_get_level_tiling(self._h, level, ctypes.byref(w), ctypes.byref(z), ctypes.byref(n)),
              "amss_engine_get_level_tiling")
        return w.value, z.value, n.value

    def run_graph(self, level, dt, nsteps, replays=1):
        check(lib().amss_engine_run_graph(self._h, level, dt, nsteps, replays), "amss_engine_run_graph")

    def constraint_norms(self, level, first_patch=False):
        """L2 norms of the Hamiltonian, momentum (x, y, z) and Gamma (x, y, z)
        constraints and of Theta (Z4c; 0 for BSSN) of a level's current state
        (Parallel::L2Norm, Parallel.C:4214-4243), as a float64 array of 8.
        Over every patch of the level, or with first_patch over its first
        patch only, as the reference's Constraint_Out takes them."""
        out = np.zeros(8)
        fn = lib().amss_engine_constraint_norms_first_patch if first_patch else lib().amss_engine_constraint_norms
        check(fn(self._h, level, out.ctypes.data_as(_DP)), "amss_engine_constraint_norms")
        return out

    def constraint_sums(self, level):
        """The squared sums behind constraint_norms over this engine's own
        blocks (the ranks of a job add them, then take square roots)."""
        out = np.zeros(8)
        check(lib().amss_engine_constraint_sums(self._h, level, out.ctypes.data_as(_DP)),
              "amss_engine_constraint_sums")
        return out

    def psi4(self, level):
        """Psi4 of a level's current state (bssn_class::Compute_Psi4 with
        getnp4), kept on the device until the next step."""
        check(lib().amss_engine_psi4(self._h, level), "amss_engine_psi4")

    def get_psi4(self, block):
        """(Rpsi4, Ipsi4) of one block after psi4(): (2, ez, ey, ex)."""
        ex = self.blocks[block]
        out = np.empty((2, ex[2], ex[1], ex[0]))
        check(lib().amss_engine_get_psi4(self._h, block, out.ctypes.data_as(_DP)), "amss_engine_get_psi4")
        return out

    def psi4_modes(self, level, rex, nquarter=40, maxl=8):
        """surface_integral::surf_Wave after psi4(): the spin-weight -2 modes
        (l = 2..maxl, m = -l..l) of Psi4 on the sphere of radius rex, as two
        arrays (RP, IP)."""
        nn = (maxl + 1) ** 2 - 4
        rp, ip = np.zeros(nn), np.zeros(nn)
        check(lib().amss_engine_psi4_modes(self._h, level, float(rex), int(nquarter), int(maxl),
                                           rp.ctypes.data_as(_DP), ip.ctypes.data_as(_DP)), "amss_engine_psi4_modes")
        return rp, ip

    def adm_integrals(self, level, rex, nquarter=40):
        """surface_integral::surf_MassPAng: (mass, Px, Py, Pz, Sx, Sy, Sz)
        through the sphere of radius rex on a level."""
        out = np.zeros(7)
        check(lib().amss_engine_adm_integrals(self._h, level, float(rex), int(nquarter), out.ctypes.data_as(_DP)),
              "amss_engine_adm_integrals")
        return out

    def interp_points(self, level, points, fields, soa=None):
        """Values of state fields at points of a level (Parallel::PatList_Interp_Points,
        Parallel.C:5614-5667): points (n, 3), fields a list of state indices,
        soa their parities (nvar, 3) or None for all +1.  Returns
        (values (n, nvar), found (n,) bool); points outside every patch of
        the level are not found and read 0."""
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        fl = np.ascontiguousarray(fields, dtype=np.int32).reshape(-1)
        out = np.zeros((pts.shape[0], fl.size))
        found = np.zeros(pts.shape[0], dtype=np.int32)
        sp = None
        if soa is not None:
            sa = np.ascontiguousarray(soa, dtype=np.float64).reshape(fl.size, 3)
            sp = sa.ctypes.data_as(_DP)
        check(lib().amss_engine_interp_points(self._h, level, pts.shape[0], pts.ctypes.data_as(_DP), fl.size,
                                              fl.ctypes.data_as(_IP), sp, out.ctypes.data_as(_DP),
                                              found.ctypes.data_as(_IP)), "amss_engine_interp_points")
        return out, found.astype(bool)

    def set_punctures(self, positions):
        """Track punctures (n, 3) on the finest level from now on (FP64 engines)."""
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        self._ntrack = pos.shape[0]
        check(lib().amss_engine_set_punctures(self._h, pos.shape[0], pos.ctypes.data_as(_DP)),
              "amss_engine_set_punctures")

    def punctures(self):
        """The tracked positions (n, 3) after the steps issued so far."""
        out = np.zeros((self._ntrack, 3))
        check(lib().amss_engine_get_punctures(self._h, out.ctypes.data_as(_DP)), "amss_engine_get_punctures")
        return out

    def sync(self):
        """Waits for the engine's stream; returns 1 if a NaN was seen."""
        return check(lib().amss_engine_sync(self._h), "amss_engine_sync")

    @property
    def stream(self):
        return lib().amss_engine_stream(self._h)

    @property
    def launches(self):
        return lib().amss_engine_launch_count(self._h)
