"""One domain cut into x strips, as the reference cuts the domain into clusters along x
(pic2d_ParticleExchange.f90:3-1762 moves the particles between neighbouring clusters, GATHER_*_CHARGE_DENSITY
pic2d_ElectronDynamics.f90:1645-1800 sums the densities of the nodes they share, and the field of the whole domain
reaches every cluster).

A strip is a context of its own columns plus `ghost` columns on each side that faces another strip (edp_set_strip;
a side on the domain's wall has none). Next to the strips runs a context of the whole grid that only solves the
field. A step, in the order of pic2d_MainProgram.f90:151-309:
1. every strip adds its fixed-point densities into the whole grid's density (summed over the ranks: int64, exact);
2. the whole grid solves the field (FFT_X, or CG with the multigrid preconditioner for walled domains), and every
   strip copies its columns of E and of the ions' accumulated E;
3. every strip pushes, collides and ends the step;
4. the particles that ended the step in ghost columns move to the neighbour owning them, as records of 8 doubles
   (the counts first, then the records). Their charge stays where the sender deposited it.
The densities are integer sums and the particles keep their FP32 offsets, ids and tags, so a run over strips repeats
the one-context run bit for bit, ionisation aside (its new ids depend on the order of creation).

`LocalStrips` runs all strips of a domain in one process (one GPU); `StripRank` is one rank's strip, with the sums
and moves through torch.distributed (NCCL between GPUs, or gloo).
"""
import ctypes as C

import numpy as np

from . import PREC_MIXED, WARM_PREVIOUS, Simulation
from .cluster import ID_SPACE, _Buffer

REC = 8   # doubles per record: x, y (local cells), vx, vy, vz, id, tag, 0


def partition(ncx, n_strips):
    """(first own column, own columns) of each strip: ncx split as evenly as possible."""
    base, extra = divmod(int(ncx), int(n_strips))
    if base < 1:
        raise ValueError("more strips than columns")
    out, x0 = [], 0
    for r in range(n_strips):
        w = base + (1 if r < extra else 0)
        out.append((x0, w))
        x0 += w
    return out


def frames(parts, ghost, periodic):
    """(ghost columns on the left, on the right, global column of local column 0) of each strip: no ghost columns
    on a side that is the wall of a walled domain."""
    n = len(parts)
    out = []
    for r, (x0, _) in enumerate(parts):
        gl = ghost if periodic or r > 0 else 0
        gr = ghost if periodic or r < n - 1 else 0
        out.append((gl, gr, x0 - gl))
    return out


def split_particles(x, parts, x_firsts):
    """For global positions x: the strip owning each particle and its local x."""
    x = np.asarray(x, dtype=np.float64)
    starts = np.array([p[0] for p in parts])
    owner = np.searchsorted(starts, np.floor(x), side="right") - 1
    local = x - np.asarray(x_firsts)[owner]
    return owner, local


def shift(x_first_from, x_first_to, wrap, ncx):
    """x shift of a record from one strip's columns to another's; wrap = +1 / -1 when it crosses the periodic
    boundary to the right / left."""
    return float(x_first_from - x_first_to - wrap * ncx)


class Strip:
    """One strip context and the context of the whole grid whose field it uses (shared by the strips of one
    process)."""

    def __init__(self, deck, n_strips, index, ghost=4, field=None, sort_every=None, seed=None, capacity=None,
                 fuse_collisions=True, id_base=None):
        self.field = field if field is not None else Simulation(deck, PREC_MIXED, sort_every=0, seed=seed)
        p = self.field.params
        self.ncx, self.ncy = p.ncx, p.ncy
        self.periodic = bool(p.periodic_x)
        self.nx_global = p.ncx if self.periodic else p.ncx + 1   # node columns of the whole grid's arrays
        self.parts = partition(p.ncx, n_strips)
        self.frames = frames(self.parts, int(ghost), self.periodic)
        self.n_strips, self.index, self.ghost = n_strips, index, int(ghost)
        self.x0, self.own = self.parts[index]
        if self.own <= self.ghost:
            raise ValueError("each strip needs more own columns than ghost columns")
        gl, gr, self.x_first = self.frames[index]
        self.sim = Simulation(deck, PREC_MIXED, sort_every=sort_every, seed=seed, capacity=capacity,
                              fuse_collisions=fuse_collisions, strip=(self.own, gl, gr, self.x_first))
        if id_base is not None:
            self.sim.set_id_base(*id_base) if isinstance(id_base, tuple) else self.sim.set_id_base(id_base)
        self.nspec = 1 + p.n_ion_species
        self.lib = self.sim.lib
        self._bufs = {}

    # ----------------------------------------------------------------------------- particles
    def load(self, species, x, y, vx, vy, vz, ids, tags=None):
        """Uploads the particles of `species` (global positions) that this strip owns."""
        owner, local = split_particles(x, self.parts, [f[2] for f in self.frames])
        m = owner == self.index
        self.sim.upload_particles(species, local[m], np.asarray(y)[m], np.asarray(vx)[m], np.asarray(vy)[m],
                                  np.asarray(vz)[m], ids=np.asarray(ids, dtype=np.uint32)[m],
                                  tag=None if tags is None else np.asarray(tags, dtype=np.int32)[m])

    def download(self, species):
        """The strip's particles of `species` with global x in [0, ncx)."""
        d = self.sim.download_particles(species)
        d["x"] = d["x"] + self.x_first
        if self.periodic:
            d["x"] = np.mod(d["x"], self.ncx)
        return d

    def shifts(self):
        """x shifts of the records sent to the left and to the right neighbour (their local columns)."""
        r, n = self.index, self.n_strips
        lo, hi = (r - 1) % n, (r + 1) % n
        return (shift(self.x_first, self.frames[lo][2], -1 if r == 0 else 0, self.ncx),
                shift(self.x_first, self.frames[hi][2], 1 if r == n - 1 else 0, self.ncx))

    # ----------------------------------------------------------------------------- one step
    def add_density(self):
        """Adds the strip's densities into the whole grid's (edp_strip_add_density), on the strip's stream."""
        for s in range(self.nspec):
            ptr, _ = self.field.device_buffer(0, s)
            self.sim._check(self.lib.edp_strip_add_density(self.sim.ctx, s, C.c_void_p(ptr), self.nx_global,
                                                           self.x_first), "edp_strip_add_density")

    def set_field(self):
        e, _ = self.field.device_buffer(1)
        a, _ = self.field.device_buffer(2)
        self.sim._check(self.lib.edp_strip_set_field(self.sim.ctx, C.c_void_p(e), C.c_void_p(a), self.nx_global,
                                                     self.x_first), "edp_strip_set_field")

    def advance(self):
        """ADVANCE_ELECTRONS, ADVANCE_IONS, the collisions and the end of the step on the strip."""
        lib, ctx, chk = self.lib, self.sim.ctx, self.sim._check
        chk(lib.edp_advance_electrons(ctx), "edp_advance_electrons")
        chk(lib.edp_advance_ions(ctx), "edp_advance_ions")
        chk(lib.edp_collide_en(ctx, None), "edp_collide_en")
        chk(lib.edp_collide_rcx(ctx, None), "edp_collide_rcx")
        chk(lib.edp_end_ion_cycle(ctx), "edp_end_ion_cycle")

    def _buffer(self, species, side, cap):
        import torch
        key = (species, side)
        b = self._bufs.get(key)
        if b is None or b.shape[0] < cap:
            b = torch.empty((cap, REC), dtype=torch.float64, device="cuda")
            self._bufs[key] = b
        return b

    def take(self, species):
        """(left records, right records) of the particles of `species` in the ghost columns, device tensors; the
        particles leave the strip."""
        c = self.sim.counters()
        live = int(c.n_particles[species])
        cap = live * 2 * (self.ghost + 1) // self.own + 65536
        left, right = self._buffer(species, 0, cap), self._buffer(species, 1, cap)
        nl, nr = C.c_int64(), C.c_int64()
        rc = self.lib.edp_strip_take(self.sim.ctx, species, C.c_void_p(left.data_ptr()), left.shape[0],
                                     C.c_void_p(right.data_ptr()), right.shape[0], C.byref(nl), C.byref(nr))
        if rc == -3 and (nl.value > left.shape[0] or nr.value > right.shape[0]):
            # the particles past the buffers stayed in the strip: keep the records taken, take the rest
            got_l, got_r = left[:min(nl.value, left.shape[0])].clone(), right[:min(nr.value, right.shape[0])].clone()
            more_l, more_r = self._buffer(species, 0, nl.value), self._buffer(species, 1, nr.value)
            rc = self.lib.edp_strip_take(self.sim.ctx, species, C.c_void_p(more_l.data_ptr()), more_l.shape[0],
                                         C.c_void_p(more_r.data_ptr()), more_r.shape[0], C.byref(nl), C.byref(nr))
            self.sim._check(rc, "edp_strip_take")
            import torch
            return torch.cat([got_l, more_l[:nl.value]]), torch.cat([got_r, more_r[:nr.value]])
        self.sim._check(rc, "edp_strip_take")
        return left[:nl.value], right[:nr.value]

    def put(self, species, records, shift):
        """Appends records (a device tensor [n, 8]) with x shifted by `shift` cells."""
        n = int(records.shape[0])
        if n == 0:
            return
        records = records.contiguous()
        self.sim._check(self.lib.edp_strip_put(self.sim.ctx, species, C.c_void_p(records.data_ptr()), n, shift),
                        "edp_strip_put")
        self.sim.synchronize()   # the records' memory is the caller's

    def close(self):
        self.sim.close()


def _solve_field(field, t):
    """UPDATE_WALL_POTENTIALS and the field of the whole grid, as edp_step solves it."""
    f = field
    f._check(f.lib.edp_update_wall_potentials(f.ctx, t), "edp_update_wall_potentials")
    if f.periodic:
        f.solve_poisson_fftx_linsysy()
    else:
        it = C.c_int32()
        f._check(f.lib.edp_field_cg(f.ctx, 1e-8, 100000, WARM_PREVIOUS, C.byref(it)), "edp_field_cg")
    f.synchronize()


def _zero_field_density(field, nspec):
    import torch
    for s in range(nspec):
        ptr, n = field.device_buffer(0, s)
        torch.as_tensor(_Buffer(ptr, n, True, True), device="cuda").zero_()


class LocalStrips:
    """All strips of one periodic domain in one process, with one context of the whole grid."""

    def __init__(self, deck, n_strips, ghost=4, sort_every=None, seed=None, capacity=None, fuse_collisions=True):
        self.field = Simulation(deck, PREC_MIXED, sort_every=0, seed=seed)
        self.strips = [Strip(deck, n_strips, r, ghost, self.field, sort_every, seed, capacity, fuse_collisions,
                             id_base=(r * (ID_SPACE // n_strips), (r + 1) * (ID_SPACE // n_strips)))
                       for r in range(n_strips)]
        self.nspec = self.strips[0].nspec
        self.t = 0

    def load(self, species, x, y, vx, vy, vz, ids, tags=None):
        for s in self.strips:
            s.load(species, x, y, vx, vy, vz, ids, tags)

    def download(self, species):
        parts = [s.download(species) for s in self.strips]
        return {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}

    def step(self, n=1):
        import torch
        f = self.field
        for _ in range(n):
            torch.cuda.synchronize()
            _zero_field_density(f, self.nspec)
            torch.cuda.synchronize()
            for s in self.strips:
                s.add_density()
                s.sim.synchronize()
            _solve_field(f, self.t)
            for s in self.strips:
                s.set_field()
                s.advance()
            f._check(f.lib.edp_end_ion_cycle(f.ctx), "edp_end_ion_cycle")
            f.synchronize()
            self.exchange()
            self.t += 1

    def exchange(self):
        k = len(self.strips)
        for sp in range(self.nspec):
            moved = [s.take(sp) for s in self.strips]
            for r, s in enumerate(self.strips):
                left, right = moved[r]
                sl, sr = s.shifts()
                self.strips[(r - 1) % k].put(sp, left, sl)
                self.strips[(r + 1) % k].put(sp, right, sr)

    def counters(self):
        """Sums of the strips' particle counts and wall hits."""
        cs = [s.sim.counters() for s in self.strips]
        return {"n_particles": [sum(c.n_particles[q] for c in cs) for q in range(self.nspec)],
                "electron_hits": [sum(c.electron_hits[q] for c in cs) for q in range(8)],
                "ion_hits": [sum(c.ion_hits[q] for c in cs) for q in range(8)]}

    def close(self):
        for s in self.strips:
            s.close()
        self.field.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class StripRank:
    """This rank's strip of a domain cut over the ranks of `group`: the density sum is an all-reduce of the
    whole-grid densities, and the moves are point-to-point sends to the two neighbours."""

    def __init__(self, deck, rank, world, ghost=4, group=None, sort_every=None, seed=None, capacity=None,
                 fuse_collisions=True):
        self.rank, self.world, self.group = rank, world, group
        self.strip = Strip(deck, world, rank, ghost, None, sort_every, seed, capacity, fuse_collisions,
                           id_base=(rank * (ID_SPACE // world), (rank + 1) * (ID_SPACE // world)))
        self.field = self.strip.field
        self.nspec = self.strip.nspec
        self.t = 0

    def step(self, n=1):
        import torch
        import torch.distributed as dist
        f, s = self.field, self.strip
        for _ in range(n):
            torch.cuda.synchronize()
            _zero_field_density(f, self.nspec)
            torch.cuda.synchronize()
            s.add_density()
            s.sim.synchronize()
            if self.world > 1:
                for sp in range(self.nspec):
                    ptr, cnt = f.device_buffer(0, sp)
                    dist.all_reduce(torch.as_tensor(_Buffer(ptr, cnt, True, True), device="cuda"), group=self.group)
                torch.cuda.synchronize()
            _solve_field(f, self.t)
            s.set_field()
            s.advance()
            f._check(f.lib.edp_end_ion_cycle(f.ctx), "edp_end_ion_cycle")
            f.synchronize()
            self.exchange()
            self.t += 1

    def exchange(self):
        """Moves the ghost-column particles to the neighbours: counts, then records (send right / receive from
        left, and the reverse), through batched point-to-point operations."""
        import torch
        import torch.distributed as dist
        for sp in range(self.nspec):
            left, right = self.strip.take(sp)
            sl, sr = self.strip.shifts()
            if self.world == 1:
                self.strip.put(sp, left, sl)
                self.strip.put(sp, right, sr)
                continue
            if dist.get_backend(self.group) == "gloo":   # gloo moves host tensors point to point
                left, right = left.cpu(), right.cpu()
            from_left, from_right = exchange_records(left, right, self.rank, self.world, self.group)
            # what comes from a neighbour was its ghost column on this side: shift from its columns into ours
            st, r, n = self.strip, self.rank, self.world
            lo, hi = (r - 1) % n, (r + 1) % n
            self.strip.put(sp, from_left.to("cuda"), shift(st.frames[lo][2], st.x_first, 1 if r == 0 else 0, st.ncx))
            self.strip.put(sp, from_right.to("cuda"), shift(st.frames[hi][2], st.x_first, -1 if r == n - 1 else 0,
                                                            st.ncx))
            torch.cuda.synchronize()

    def close(self):
        self.strip.close()
        self.field.close()


def exchange_records(left, right, rank, world, group=None):
    """Sends `left` to rank - 1 and `right` to rank + 1 (periodic) and returns (records from the left neighbour,
    records from the right neighbour). Counts travel first; records of 8 doubles follow. Works on CPU tensors
    (gloo) and on device tensors (NCCL)."""
    import torch
    import torch.distributed as dist
    dev = left.device
    lo, hi = (rank - 1) % world, (rank + 1) % world
    n_out = torch.tensor([left.shape[0], right.shape[0]], dtype=torch.int64, device=dev)
    n_from_left = torch.zeros(1, dtype=torch.int64, device=dev)
    n_from_right = torch.zeros(1, dtype=torch.int64, device=dev)
    # the same order on every rank (right before left, from the left before from the right): with two ranks both
    # neighbours are one rank, and the operations between a pair match in the order they are posted
    ops = [dist.P2POp(dist.isend, n_out[1:2].clone(), hi, group), dist.P2POp(dist.isend, n_out[0:1].clone(), lo, group),
           dist.P2POp(dist.irecv, n_from_left, lo, group), dist.P2POp(dist.irecv, n_from_right, hi, group)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()
    a, b = int(n_from_left.item()), int(n_from_right.item())
    from_left = torch.empty((a, REC), dtype=torch.float64, device=dev)
    from_right = torch.empty((b, REC), dtype=torch.float64, device=dev)
    ops = []
    if right.shape[0]:
        ops.append(dist.P2POp(dist.isend, right.contiguous(), hi, group))
    if left.shape[0]:
        ops.append(dist.P2POp(dist.isend, left.contiguous(), lo, group))
    if a:
        ops.append(dist.P2POp(dist.irecv, from_left, lo, group))
    if b:
        ops.append(dist.P2POp(dist.irecv, from_right, hi, group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    return from_left, from_right
