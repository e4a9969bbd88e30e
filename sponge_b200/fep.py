"""FEP/TI windows: one soft-core system per lambda, and many of them batched on one GPU.

``FepEngine(system)`` wires NEIGHBOR_LIST, LJ_SOFT_CORE and Particle_Mesh_Ewald for one box of
``sponge_b200.systems.fep_box`` (the charges at the box's lambda, their change per unit lambda,
A/B LJ types and tables, the perturbation mask). ``step()`` is one force evaluation with
dU/dlambda (``sb_fep_step``: soft-core LJ + direct, exclusion correction, reciprocal space, PME
cross terms and the long-range correction, no host synchronisation).

``FepBatch(systems)`` runs many such boxes of uneven size together. Each box keeps its own
modules and list. In the default mode (``mode="kernels"``) one force step of all boxes is
``sb_fep_batch_step``: one launch per stage over all boxes' slots, clusters and atoms through
per-box descriptors, plus one launch per FFT stage per group of equal grid sizes; the step is
captured once as a CUDA graph. ``mode="streams"`` keeps each box's own ``sb_fep_step`` launches
as concurrent branches of one graph, spread over a tuned number of streams. Both give every box
the bits of its own step. List rebuilds run between replays.
"""

import numpy as np

from . import (FORM_FIXED, FepBatchStep, NeighborList, ParticleMeshEwald, SoftCore,
               _require_cuda, crd_to_uint_crd, fep_step, pme_ti_cross)


def _scaled(x, f):
    return (np.asarray(x, np.float32) * np.float32(f)).astype(np.float32)


class FepEngine:
    def __init__(self, system, form=FORM_FIXED, refresh_interval=20, max_neighbor_numbers=1200,
                 device="cuda", prune_buffer=0.5, prune_interval=0):
        torch = _require_cuda()
        self.torch = torch
        self.system = s = system
        self.n = n = len(s["charge"])
        self.box = np.asarray(s["box"], np.float32)
        dev = torch.device(device)
        self.crd = torch.tensor(np.asarray(s["crd"], np.float32), device=dev)
        self.charge = torch.tensor(np.asarray(s["charge"], np.float32), device=dev)
        self.dq = torch.tensor(np.asarray(s["dq"], np.float32), device=dev)
        self.excl_start = torch.tensor(s["excl_start"], dtype=torch.int32, device=dev)
        self.excl_numbers = torch.tensor(s["excl_numbers"], dtype=torch.int32, device=dev)
        el = s["excl_list"] if len(s["excl_list"]) else np.zeros(1, np.int32)
        self.excl_list = torch.tensor(el, dtype=torch.int32, device=dev)
        self.uint_crd = torch.empty((n, 3), dtype=torch.int32, device=dev)
        self.frc = torch.zeros((n, 3), dtype=torch.float32, device=dev)
        self.dudl = torch.zeros(1, dtype=torch.float64, device=dev)
        self.nl = NeighborList(n, self.box, s["cutoff"], s["skin"], refresh_interval,
                               max_neighbor_numbers=max_neighbor_numbers, form=form)
        self.sc = SoftCore(n, _scaled(s["lj_A"], 12), _scaled(s["lj_B"], 6),
                           _scaled(s["lj_A_B"], 12), _scaled(s["lj_B_B"], 6), s["lj_type"],
                           s["lj_type_B"], s["mask"], s["dq"], s["cutoff"], self.box, s["lam"],
                           s["sc_alpha"], s["sc_p"], s["sc_sigma"], s["sc_sigma_min"], form=form,
                           n_types_A=s["n_types"], n_types_B=s["n_types_B"])
        self.pme = ParticleMeshEwald(n, self.box, s["cutoff"], s["tolerance"], s["fft"],
                                     form=form)
        # the split form's packed pair kernel walks a pruned list (rc + prune_buffer, pruned
        # again after a rebuild and when an atom has moved half the buffer); 0.5 A suits steps on
        # fixed coordinates, while MD at 300 K runs faster with 1 A (fewer prunes)
        if form == FORM_FIXED and prune_buffer > 0 and self.sc.split_form[0]:
            self.nl.set_prune(prune_buffer, prune_interval)
        self.scaler = (np.float32(1.0) / np.float32(4294967296.0)) * self.box
        self.form = form

    @property
    def excl(self):
        return (self.excl_start, self.excl_list, self.excl_numbers)

    def update_list(self, forced=0, stream=None):
        self.nl.Neighbor_List_Update(self.crd, self.excl_start, self.excl_list, self.excl_numbers,
                                     forced_update=forced, stream=stream)

    def to_uint(self, stream=None):
        crd_to_uint_crd(self.crd, self.box, out=self.uint_crd, stream=stream)

    def step(self, want_dudl=True, stream=None):
        """Fused fixed-form FEP force step (forces += into self.frc, dU/dlambda to self.dudl)."""
        fep_step(self.nl, self.sc, self.pme, self.uint_crd, self.charge, self.excl, self.frc,
                 self.dudl if want_dudl else None, stream=stream)

    def forces_modules(self, stream=None):
        """The module-by-module sequence (either form): soft-core LJ + direct, exclusion
        correction, reciprocal space, forces += into self.frc."""
        self.sc.LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial(
            self.n, self.uint_crd, self.charge, self.frc, self.nl, self.pme.beta, stream=stream)
        self.pme.PME_Excluded_Force_With_Atom_Energy(
            self.uint_crd, self.scaler, self.charge, self.excl_start, self.excl_list,
            self.excl_numbers, self.frc, self.pme.d_correction_atom_energy, stream=stream)
        self.pme.PME_Reciprocal_Force_With_Energy_And_Virial(self.uint_crd, self.charge,
                                                             self.frc, stream=stream)

    def dudl_parts(self, stream=None):
        """dU/dlambda by parts through the module calls (synchronising)."""
        lj, direct, lrc = self.sc.Get_Partial_H_Partial_Lambda(self.uint_crd, self.charge,
                                                               self.nl, self.pme.beta,
                                                               stream=stream)
        parts = dict(dhdl_lj=lj, dhdl_direct=direct, dhdl_lrc=lrc)
        if self.form == FORM_FIXED:
            rec, slf, cor = pme_ti_cross(self.pme, self.uint_crd, self.charge, self.dq,
                                         self.excl, stream=stream)
            parts.update(cross_rec=rec, cross_self=slf, cross_corr=cor)
        return parts


class FepBatch:
    """Many FEP boxes on one GPU, one captured CUDA graph per force step."""

    def __init__(self, systems, refresh_interval=20, mode="kernels"):
        torch = _require_cuda()
        if mode not in ("kernels", "streams"):
            raise ValueError("mode must be 'kernels' or 'streams'")
        self.torch = torch
        self.mode = mode
        self.engines = [FepEngine(s, refresh_interval=refresh_interval) for s in systems]
        self.refresh_interval = refresh_interval
        self.dudl = torch.zeros(len(self.engines), dtype=torch.float64, device="cuda")
        # one force array for all boxes: a single clear per step
        self.frc = torch.zeros((self.atoms, 3), dtype=torch.float32, device="cuda")
        o = 0
        for k, e in enumerate(self.engines):
            e.dudl = self.dudl[k:k + 1]
            e.frc = self.frc[o:o + e.n]
            o += e.n
        self.graph = None
        self.n_streams = None
        self._batches = {}  # sub-batch count -> list of FepBatchStep
        self.count = 0

    @property
    def atoms(self):
        return sum(e.n for e in self.engines)

    @property
    def launches(self):
        """Kernel launches of one captured step (the force clear included)."""
        if self.mode == "kernels" and self.n_streams in self._batches:
            return 1 + sum(b.launches for b in self._batches[self.n_streams])
        return None

    def _rebuild_all(self, n_streams):
        torch = self.torch
        if getattr(self, "_rb_streams", None) is None or len(self._rb_streams) != n_streams:
            self._rb_streams = [torch.cuda.Stream() for _ in range(n_streams)]
        cur = torch.cuda.current_stream()
        for st in self._rb_streams:
            st.wait_stream(cur)
        for k, e in enumerate(self.engines):
            st = self._rb_streams[k % n_streams]
            with torch.cuda.stream(st):
                e.update_list(forced=1, stream=st)
                e.to_uint(stream=st)
        for st in self._rb_streams:
            cur.wait_stream(st)

    def rebuild(self, n_streams=8):
        """List rebuild of every box (a forced update: no host synchronisation), the boxes spread
        over n_streams streams. The first call runs eagerly and captures the same launches as a
        CUDA graph, which the later calls replay (the host would otherwise spend longer issuing
        the seven launches of each box than the device spends running them)."""
        torch = self.torch
        if getattr(self, "_rb_graph", None) is not None:
            self._rb_graph.replay()
            return
        self._rebuild_all(n_streams)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=torch.cuda.Stream()):
            self._rebuild_all(n_streams)
        self._rb_graph = g

    def _sub_batches(self, n):
        """The boxes in n sub-batches of balanced cost, one sb_fep_batch each."""
        if n not in self._batches:
            parts = shard_boxes([box_cost(e.system) for e in self.engines], n)
            self._batches[n] = [
                FepBatchStep([(e.nl, e.sc, e.pme, e.uint_crd, e.charge, e.excl, e.frc, e.dudl)
                              for e in (self.engines[k] for k in part)])
                for part in parts if part]
        return self._batches[n]

    def _eager_step(self, n=1):
        self.frc.zero_()
        if self.mode == "kernels":
            for b in self._sub_batches(n):
                b.step()
        else:
            for e in self.engines:
                e.step()

    def capture(self, n_streams=1):
        """Capture one force step of every box: in kernels mode n_streams sub-batches of
        batched launches, in streams mode each box's own launches, box k on stream
        k mod n_streams; the branches run concurrently."""
        torch = self.torch
        self._eager_step(n_streams)  # first calls size per-list scratch outside the capture
        torch.cuda.synchronize()
        main = torch.cuda.Stream()
        streams = [torch.cuda.Stream() for _ in range(n_streams)]
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=main):
            cur = torch.cuda.current_stream()
            self.frc.zero_()
            for st in streams:
                st.wait_stream(cur)
            if self.mode == "kernels":
                for k, b in enumerate(self._sub_batches(n_streams)):
                    b.step(stream=streams[k])
            else:
                for k, e in enumerate(self.engines):
                    e.step(stream=streams[k % n_streams])
            for st in streams:
                cur.wait_stream(st)
        self.graph = g
        self.n_streams = n_streams
        self._streams = (main, streams)
        return g

    def step(self):
        """One step of all boxes: list rebuild every refresh_interval steps, then the graph."""
        if self.count % self.refresh_interval == 0:
            self.rebuild()
        self.graph.replay()
        self.count += 1

    def _replay_ms(self, reps):
        torch = self.torch
        for _ in range(2):
            self.graph.replay()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            self.graph.replay()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    def tune(self, candidates=None, reps=5):
        """Capture the step with the branch count (sub-batches in kernels mode, streams in
        streams mode) whose replay is fastest. Returns (count, ms per replay)."""
        if candidates is None:
            candidates = (1, 2, 3, 4, 6) if self.mode == "kernels" else (1, 4, 8, 16, 48)
        best = None
        for ns in candidates:
            if ns > len(self.engines):
                continue
            self.capture(ns)
            ms = self._replay_ms(reps)
            if best is None or ms < best[1]:
                best = (ns, ms)
        self.capture(best[0])
        return best


def shard_boxes(costs, world):
    """Greedy assignment of boxes to ranks, largest first onto the least-loaded rank.
    Returns a list of box-index lists, one per rank (each sorted)."""
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for k in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(world), key=lambda j: (load[j], j))
        parts[r].append(k)
        load[r] += costs[k]
    return [sorted(p) for p in parts]


def box_cost(system):
    """Relative cost of one box's step: atoms (pair work) plus grid points (FFT work)."""
    K = system["fft"]
    return float(len(system["charge"])) + 0.25 * float(K[0] * K[1] * K[2])
