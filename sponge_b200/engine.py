"""NonbondedEngine: the three modules wired together the way SPONGE's MD driver calls them.

Main_Calculate_Force (SPONGE/main.cu:162-210) calls, in order, LJ + PME direct
(``LJ_PME_Direct_Force_With_Atom_Energy_And_Virial``), the LJ long-range correction, the PME
exclusion correction and PME reciprocal space; Main_Iteration (main.cu:376) then updates the
neighbor list. The engine owns device copies of one system's arrays (from
``sponge_b200.systems``) and exposes both the per-module sequence and the fused C entry point.
"""

import numpy as np

from . import (FORM_FIXED, LennardJones, NeighborList, ParticleMeshEwald, _require_cuda,
               crd_to_uint_crd, nonbonded_force, nonbonded_step)


def scaled_lj_tables(system):
    """The LJ module's h_LJ_A * 12 and h_LJ_B * 6 in float (Lennard_Jones_force.cu:1092-1098)."""
    A12 = (np.asarray(system["lj_A"], np.float32) * np.float32(12.0)).astype(np.float32)
    B6 = (np.asarray(system["lj_B"], np.float32) * np.float32(6.0)).astype(np.float32)
    return A12, B6


class NonbondedEngine:
    """``prune_buffer`` / ``prune_interval``: the pruned pair list of the fixed form
    (NeighborList.set_prune): the pair kernel walks the entries within cutoff + prune_buffer of
    the last prune, renewed after each rebuild and when an atom has moved half the buffer (which
    keeps every pair inside the cut-off in it), plus every ``prune_interval`` list updates when
    that is > 0 (a count only adds prunes). The default 1 A buffer is the fastest of 0.5-1.5 A
    for MD of the 96,000-atom water box at 300 K (a prune about every fourth step). A buffer of 0
    turns the pruned list off."""

    def __init__(self, system, form=FORM_FIXED, refresh_interval=20, max_neighbor_numbers=1200,
                 device="cuda", prune_buffer=1.0, prune_interval=0):
        torch = _require_cuda()
        self.torch = torch
        self.system = system
        self.n = n = int(len(system["charge"]))
        self.box = np.asarray(system["box"], np.float32)
        dev = torch.device(device)
        self.crd = torch.tensor(np.asarray(system["crd"], np.float32), device=dev)
        self.charge = torch.tensor(np.asarray(system["charge"], np.float32), device=dev)
        self.excl_start = torch.tensor(system["excl_start"], dtype=torch.int32, device=dev)
        self.excl_numbers = torch.tensor(system["excl_numbers"], dtype=torch.int32, device=dev)
        el = system["excl_list"] if len(system["excl_list"]) else np.zeros(1, np.int32)
        self.excl_list = torch.tensor(el, dtype=torch.int32, device=dev)
        self.uint_crd = torch.empty((n, 3), dtype=torch.int32, device=dev)
        A12, B6 = scaled_lj_tables(system)
        self.nl = NeighborList(n, self.box, system["cutoff"], system["skin"], refresh_interval,
                               max_neighbor_numbers=max_neighbor_numbers, form=form)
        if form == FORM_FIXED and prune_buffer:
            self.nl.set_prune(min(float(prune_buffer), float(system["skin"])), prune_interval)
        self.lj = LennardJones(n, system["n_types"], A12, B6, system["lj_type"],
                               system["cutoff"], self.box, form=form)
        fft = system.get("fft") or (-1, -1, -1)
        self.pme = ParticleMeshEwald(n, self.box, system["cutoff"], system["tolerance"], fft,
                                     form=form)
        self.frc = torch.zeros((n, 3), dtype=torch.float32, device=dev)
        self.atom_energy = torch.zeros(n, dtype=torch.float32, device=dev)
        self.atom_virial = torch.zeros(n, dtype=torch.float32, device=dev)
        self.d_virial = torch.zeros(1, dtype=torch.float32, device=dev)
        self.d_potential = torch.zeros(1, dtype=torch.float32, device=dev)
        self.scaler = (np.float32(1.0) / np.float32(4294967296.0)) * self.box
        self._graph = None
        self._md_graph = None

    @property
    def excl(self):
        return (self.excl_start, self.excl_list, self.excl_numbers)

    def update_list(self, forced=0, stream=None):
        self.nl.Neighbor_List_Update(self.crd, self.excl_start, self.excl_list, self.excl_numbers,
                                     forced_update=forced, stream=stream)

    def to_uint(self, stream=None):
        crd_to_uint_crd(self.crd, self.box, out=self.uint_crd, stream=stream)

    def reset(self):
        self.frc.zero_()
        self.atom_energy.zero_()
        self.atom_virial.zero_()
        self.d_virial.zero_()
        self.d_potential.zero_()

    def forces(self, need_energy=0, need_virial=0, parts=("direct", "lrc", "excluded",
                                                          "reciprocal"), stream=None):
        """Module-by-module force evaluation (adds into self.frc)."""
        if "direct" in parts:
            self.lj.LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(
                self.n, self.uint_crd, self.charge, self.frc, self.nl, self.pme.beta,
                need_energy, self.atom_energy, need_virial, self.atom_virial,
                self.pme.d_direct_atom_energy, stream=stream)
        if "lrc" in parts:
            self.lj.Long_Range_Correction(need_virial, self.d_virial, need_energy,
                                          self.d_potential, stream=stream)
        if "excluded" in parts:
            self.pme.PME_Excluded_Force_With_Atom_Energy(
                self.uint_crd, self.scaler, self.charge, self.excl_start, self.excl_list,
                self.excl_numbers, self.frc, self.pme.d_correction_atom_energy, stream=stream)
        if "reciprocal" in parts:
            self.pme.PME_Reciprocal_Force_With_Energy_And_Virial(
                self.uint_crd, self.charge, self.frc, need_virial, need_energy, self.d_virial,
                self.d_potential, stream=stream)

    def step(self, need_energy=0, need_virial=0, stream=None):
        """Fused C entry point: list update by policy + all force terms."""
        nonbonded_step(self.nl, self.lj, self.pme, self.crd, self.uint_crd, self.charge,
                       self.excl, self.frc, need_energy, need_virial, self.atom_energy,
                       self.atom_virial, self.d_virial, self.d_potential, stream=stream)

    def force(self, need_energy=0, need_virial=0, stream=None):
        """Force part only, list as it stands (sb_nonbonded_force)."""
        nonbonded_force(self.nl, self.lj, self.pme, self.uint_crd, self.charge, self.excl,
                        self.frc, need_energy, need_virial, self.atom_energy, self.atom_virial,
                        self.d_virial, self.d_potential, stream=stream)

    def update_box(self, box_length):
        """Box change as Main_Box_Length_Change / Main_Volume_Change call it (SPONGE/main.cu:438-460)
        after the caller has scaled the coordinates: NEIGHBOR_LIST::Update_Volume (the next list
        update rebuilds), LENNARD_JONES_INFORMATION::Update_Volume and
        Particle_Mesh_Ewald::Update_Box_Length. Captured graphs hold the old box's scale factors
        as kernel arguments, so they are dropped here and captured again at their next replay."""
        box = np.asarray(box_length, np.float32).reshape(3)
        self.nl.Update_Volume(box)
        self.lj.Update_Volume(box)
        self.pme.Update_Box_Length(box)
        self.box = box
        self.scaler = (np.float32(1.0) / np.float32(4294967296.0)) * self.box
        self._graph = None
        self._md_graph = None

    def capture_force_graph(self):
        """Capture (frc = 0; force part) once as a CUDA graph; ``step_graph`` replays it after
        the list update by its policy. Call once eagerly first (lazy per-list buffers). A box
        change (``update_box``) drops the graph; ``step_graph`` then captures it again."""
        torch = self.torch
        self.frc.zero_()
        self.force()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream()
        with torch.cuda.graph(g, stream=side):
            self.frc.zero_()
            self.force()
        self._graph = g
        return g

    def step_graph(self):
        """List update by its policy (eager), then the captured force graph (captured again
        first when the box changed since the last capture)."""
        self.update_list()
        if self._graph is None:
            self.capture_force_graph()
        self._graph.replay()

    def md_step(self, settle, inverse_mass, mass, vel, acc=None):
        """One NVE step as Main_Calculate_Force + Main_Iteration run it (SPONGE/main.cu:162-329,
        :376), eagerly: fixed-point coordinates, forces (list as it stands), then the fused
        leap-frog + SETTLE launch (``settle``: a Settle handle with no constraint pairs left)."""
        crd_to_uint_crd(self.crd, self.box, out=self.uint_crd)
        self.frc.zero_()
        self.force()
        settle.nve_step(self.uint_crd, self.scaler, inverse_mass, mass, self.frc, vel, self.crd,
                        self.box, acc=acc)

    def capture_md_graph(self, settle, inverse_mass, mass, vel, acc=None):
        """Capture ``md_step`` once as a CUDA graph (the integrator and SETTLE behind the force
        graph); ``md_step_graph`` replays it after the list update by its policy. The buffers
        passed here are the ones every replay uses. Call ``md_step`` once eagerly first (lazy
        per-list buffers)."""
        torch = self.torch
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream()
        with torch.cuda.graph(g, stream=side):
            self.md_step(settle, inverse_mass, mass, vel, acc)
        self._md_graph = g
        self._md_args = (settle, inverse_mass, mass, vel, acc)
        return g

    def md_step_graph(self):
        """List update by its policy (eager, wraps the coordinates on rebuilds), then the captured
        MD step (captured again, with the buffers of the last capture, after a box change)."""
        self.update_list()
        if self._md_graph is None:
            self.md_step(*self._md_args)
            self.capture_md_graph(*self._md_args)
            return
        self._md_graph.replay()

    def potential(self):
        """Total potential as MD_core sums it: sum(atom_energy) + d_potential (FP64 sum)."""
        return float(self.atom_energy.double().sum().item() + self.d_potential.double().item())

    def virial(self):
        return float(self.atom_virial.double().sum().item() + self.d_virial.double().item())
