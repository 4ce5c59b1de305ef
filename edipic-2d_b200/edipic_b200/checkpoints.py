"""Checkpoints in the reference's file layouts, so that a device run can continue a CPU run and the reverse.

* POSIX (SAVE_CHECKPOINT_POSIX / READ_CHECKPOINT_POSIX, pic2d_Checkpoints.f90:702-1124): one stream file per MPI
  rank, `checkdir_TTTTTTTT/Tcntr_TTTTTTTT_proc_PPP.check`, holding that rank's header (INTEGER), surface charges
  (REAL(8)), then its electrons and the ions of each species as records X, Y, VX, VY, VZ (REAL(8)), tag (INTEGER).
* MPI-IO (SAVE_CHECKPOINT_MPIIO_2 / READ_CHECKPOINT_MPIIO_2, :5-660): one file `Tcntr_TTTTTTTT.check` written with
  MPI_FILE_WRITE_ORDERED, so each block is the concatenation over ranks in rank order: the headers, the surface
  charges, the electrons' (X, Y, VX, VY, VZ) rows, the electrons' tags, then the same two blocks per ion species.

The header of a rank (INTEGER, 1-based as in the reference): 1-624 the WELL19937a state, 625 its index, 626 its
case function, 627 T_cntr, 628/629 the load-balance counters, 630 Save_probes_e_data_T_cntr, 631 N_of_saved_records,
632 current_snap, 633 particle_master, 634 max_N_electrons, 635 N_electrons, 636 total_cathode_N_e_to_inject, then
max_N_ions(s), N_ions(s) per species and last len_surf_charge. Values are in the machine's byte order.

The device keeps no WELL19937a stream (its variates are counter-based, keyed by particle id and step), so a checkpoint
written here carries either the RNG states of the checkpoint the run was loaded from, or per-rank states seeded as
well_random_seed (pic2d_RandomNumberInterface.f90:39-57) does. The surface charges of dielectric inner objects are
rank 0's REAL(8) block, each object's outline in the order of its boundary nodes (pic2d_Checkpoints.f90:806-812);
dielectric walls and object potentials (external circuits) are outside the device path and rejected on loading.
"""
import os

import numpy as np

REC = np.dtype([("x", "<f8"), ("y", "<f8"), ("vx", "<f8"), ("vy", "<f8"), ("vz", "<f8"), ("tag", "<i4")])
ROW = np.dtype([("x", "<f8"), ("y", "<f8"), ("vx", "<f8"), ("vy", "<f8"), ("vz", "<f8")])
H_STATE, H_IND, H_FUNC, H_TCNTR, H_GLB, H_CLB, H_PROBES, H_RECORDS, H_SNAP, H_MASTER = range(0, 624), 624, 625, 626, \
    627, 628, 629, 630, 631, 632
H_MAXNE, H_NE, H_CATHODE = 633, 634, 635


def header_length(n_spec):
    """ibufer_length = 636 + 2 N_spec + 1 (pic2d_Checkpoints.f90:748)."""
    return 636 + 2 * n_spec + 1


def well_seed_state(seed):
    """The WELL19937a state that well_random_seed(seed) sets (pic2d_RandomNumberInterface.f90:39-57): state(1) = seed,
    state(j) = 1812433253 * (state(j-1) XOR (state(j-1) << 30)) + j - 1 modulo 2^32, index 0, case function 1
    (Knuth's initialisation multiplier, TAOCP vol. 2, 3rd ed., p. 106; the shift is to the left, as ISHFT(x, 30))."""
    s = np.zeros(624, np.uint64)
    s[0] = seed & 0xFFFFFFFF
    for j in range(1, 624):
        x = int(s[j - 1])
        x ^= (x << 30) & 0xFFFFFFFF
        s[j] = (1812433253 * x + j) & 0xFFFFFFFF
    return s.astype(np.uint32).view(np.int32), 0, 1


class Rank:
    """The content of one MPI rank's part of a checkpoint."""

    def __init__(self, header, surf, electrons, ions):
        self.header = np.asarray(header, np.int32)
        self.surf = np.asarray(surf, np.float64)
        self.electrons = electrons          # structured array, REC fields
        self.ions = list(ions)              # one structured array per ion species

    @property
    def t_cntr(self):
        return int(self.header[H_TCNTR])

    def rng(self):
        return self.header[:624].copy(), int(self.header[H_IND]), int(self.header[H_FUNC])


def _counts(header, n_spec):
    ne = int(header[H_NE])
    ni = [int(header[637 - 1 + 2 * s + 1]) for s in range(n_spec)]
    return ne, ni, int(header[header_length(n_spec) - 1])


def posix_path(root, t_cntr, rank):
    return os.path.join(root, f"checkdir_{t_cntr:08d}", f"Tcntr_{t_cntr:08d}_proc_{rank:03d}.check")


def mpiio_path(root, t_cntr):
    return os.path.join(root, f"Tcntr_{t_cntr:08d}.check")


def read_posix(root, t_cntr, n_spec):
    """All ranks' files of a POSIX checkpoint (proc_000, proc_001, ... until the first missing one)."""
    ranks = []
    while os.path.exists(posix_path(root, t_cntr, len(ranks))):
        raw = open(posix_path(root, t_cntr, len(ranks)), "rb").read()
        L = header_length(n_spec)
        h = np.frombuffer(raw, np.int32, L)
        ne, ni, ls = _counts(h, n_spec)
        pos = 4 * L
        surf = np.frombuffer(raw, np.float64, ls, pos)
        pos += 8 * ls
        el = np.frombuffer(raw, REC, ne, pos)
        pos += REC.itemsize * ne
        ions = []
        for n in ni:
            ions.append(np.frombuffer(raw, REC, n, pos))
            pos += REC.itemsize * n
        if pos != len(raw):
            raise ValueError(f"{posix_path(root, t_cntr, len(ranks))}: {len(raw) - pos} bytes left over")
        ranks.append(Rank(h, surf, el, ions))
    if not ranks:
        raise FileNotFoundError(posix_path(root, t_cntr, 0))
    return ranks


def write_posix(root, t_cntr, ranks):
    """One file per rank in checkdir_TTTTTTTT (created if missing)."""
    os.makedirs(os.path.dirname(posix_path(root, t_cntr, 0)), exist_ok=True)
    paths = []
    for r, rk in enumerate(ranks):
        path = posix_path(root, t_cntr, r)
        with open(path, "wb") as f:
            f.write(np.ascontiguousarray(rk.header, np.int32).tobytes())
            f.write(np.ascontiguousarray(rk.surf, np.float64).tobytes())
            f.write(np.ascontiguousarray(rk.electrons, REC).tobytes())
            for a in rk.ions:
                f.write(np.ascontiguousarray(a, REC).tobytes())
        paths.append(path)
    return paths


def _mpiio_size(headers, n_spec):
    L = header_length(n_spec)
    size = 4 * L * len(headers)
    for h in headers:
        ne, ni, ls = _counts(h, n_spec)
        size += 8 * ls + (40 + 4) * ne + sum((40 + 4) * n for n in ni)
    return size


def read_mpiio(path, n_spec):
    """An MPI-IO checkpoint. The file does not store the number of ranks: it is the one whose headers agree on
    T_cntr and account for the file's size exactly."""
    raw = open(path, "rb").read()
    L = header_length(n_spec)
    heads = []
    nranks = None
    for p in range(1, len(raw) // (4 * L) + 1):
        h = np.frombuffer(raw, np.int32, L, 4 * L * (p - 1))
        if heads and h[H_TCNTR] != heads[0][H_TCNTR]:
            break
        ne, ni, ls = _counts(h, n_spec)
        if min([ne, ls] + ni) < 0:
            break
        heads.append(h)
        if _mpiio_size(heads, n_spec) == len(raw):
            nranks = p
            break
    if nranks is None:
        raise ValueError(f"{path}: no rank count matches the file size")
    pos = 4 * L * nranks
    cnt = [_counts(h, n_spec) for h in heads]
    surf = []
    for ne, ni, ls in cnt:
        surf.append(np.frombuffer(raw, np.float64, ls, pos))
        pos += 8 * ls

    def block(k):   # species k: 0 electrons, 1.. ions
        nonlocal pos
        rows, tags = [], []
        for ne, ni, _ in cnt:
            n = ne if k == 0 else ni[k - 1]
            rows.append(np.frombuffer(raw, ROW, n, pos))
            pos += ROW.itemsize * n
        for ne, ni, _ in cnt:
            n = ne if k == 0 else ni[k - 1]
            tags.append(np.frombuffer(raw, np.int32, n, pos))
            pos += 4 * n
        out = []
        for r, t in zip(rows, tags):
            a = np.zeros(len(r), REC)
            for f in ROW.names:
                a[f] = r[f]
            a["tag"] = t
            out.append(a)
        return out

    el = block(0)
    ions = [block(s + 1) for s in range(n_spec)]
    return [Rank(heads[r], surf[r], el[r], [ions[s][r] for s in range(n_spec)]) for r in range(nranks)]


def write_mpiio(path, ranks):
    """The single-file layout of SAVE_CHECKPOINT_MPIIO_2 for the given ranks."""
    n_spec = len(ranks[0].ions)
    with open(path, "wb") as f:
        for rk in ranks:
            f.write(np.ascontiguousarray(rk.header, np.int32).tobytes())
        for rk in ranks:
            f.write(np.ascontiguousarray(rk.surf, np.float64).tobytes())
        for k in range(n_spec + 1):
            parts = [rk.electrons if k == 0 else rk.ions[k - 1] for rk in ranks]
            for a in parts:
                rows = np.zeros(len(a), ROW)
                for fld in ROW.names:
                    rows[fld] = a[fld]
                f.write(rows.tobytes())
            for a in parts:
                f.write(np.ascontiguousarray(a["tag"], np.int32).tobytes())
    return path


# ------------------------------------------------------------------------------------------------- Simulation side
def outline_nodes(il, jb, ir, jt):
    """(i, j) of an inner object's boundary nodes 1..N_boundary_nodes: up the left side from (ileft, jbottom), along
    the top, down the right side, back along the bottom (Get_Surface_Charge_Inner_Object,
    pic2d_PETSc_Solver.F90:1645-1720)."""
    nodes = [(il, j) for j in range(jb, jt + 1)] + [(i, jt) for i in range(il + 1, ir + 1)]
    nodes += [(ir, j) for j in range(jt - 1, jb - 1, -1)] + [(i, jb) for i in range(ir - 1, il, -1)]
    return nodes


def _dielectrics(p):
    return [(p.inner_ileft[n], p.inner_jbottom[n], p.inner_iright[n], p.inner_jtop[n]) for n in range(p.n_inner)
            if p.inner_eps[n] > 0.0]

def _records(d):
    a = np.zeros(len(d["x"]), REC)
    for f in REC.names:
        a[f] = d[f]
    return a


def load_checkpoint(sim, t_cntr, root="."):
    """READ_A_CHECKPOINT (pic2d_Checkpoints.f90:1129-1189) into a fresh Simulation: the MPI-IO file if it exists,
    else the POSIX files. All ranks' particles are uploaded (ids follow the file order), the step counter is set
    to the saved T_cntr and the ranks are returned (their headers carry the RNG states for a later save).
    Periodic x positions in the reference's overlap cell [N, N + 1] are taken to their image in [0, 1)."""
    from . import ELECTRONS

    n_spec = sim.params.n_ion_species
    path = mpiio_path(root, t_cntr)
    ranks = read_mpiio(path, n_spec) if os.path.exists(path) else read_posix(root, t_cntr, n_spec)
    if any(rk.t_cntr != t_cntr for rk in ranks):
        raise ValueError("checkpoint T_cntr does not match its file name")
    diel = _dielectrics(sim.params)
    want = sum(len(outline_nodes(*o)) for o in diel)
    if any(len(rk.surf) for rk in ranks[1:]) or len(ranks[0].surf) != want:
        raise ValueError("checkpoint surface charges do not match the dielectric inner objects (dielectric walls or "
                         "object potentials are not supported)")
    if diel:
        from . import FIELD_SURFACE_CHARGE
        grid = np.zeros((sim.ny_ref, sim.nx_ref))
        k = 0
        for o in diel:
            for (i, j) in outline_nodes(*o):
                grid[j, i] = ranks[0].surf[k]
                k += 1
        sim.set_field(FIELD_SURFACE_CHARGE, grid)
    ncx = sim.params.ncx
    for k in range(n_spec + 1):
        a = np.concatenate([rk.electrons if k == 0 else rk.ions[k - 1] for rk in ranks])
        x = a["x"].copy()
        if sim.periodic:
            x = np.where(x >= ncx, x - ncx, x)
        if len(a):
            sim.upload_particles(ELECTRONS + k, x, a["y"], a["vx"], a["vy"], a["vz"], tag=a["tag"])
    sim.set_step(t_cntr)
    return ranks


def save_checkpoint(sim, root=".", nprocs=1, fmt="posix", carry=None, seed=1):
    """SAVE_CHECKPOINT_POSIX / SAVE_CHECKPOINT_MPIIO_2 of the device state at the start of the current step, split
    over nprocs ranks (contiguous shares of each species, rank 0 the cluster master). carry: the ranks of the
    checkpoint the run was loaded from; their RNG states and counters 628-633, 636 are written back (same nprocs).
    Without it each rank r gets the state well_random_seed(seed + r) sets and the counters start at T_cntr / 0."""
    from . import ELECTRONS

    p = sim.params
    n_spec = p.n_ion_species
    t = int(sim.counters().step)
    parts = [_records(sim.download_particles(ELECTRONS + k)) for k in range(n_spec + 1)]
    if carry is not None and len(carry) != nprocs:
        raise ValueError("carry must have one rank per process")
    ranks = []
    for r in range(nprocs):
        share = [np.array_split(a, nprocs)[r] for a in parts]
        h = np.zeros(header_length(n_spec), np.int32)
        if carry is not None:
            h[:] = carry[r].header
        else:
            st, ind, func = well_seed_state(seed + r)
            h[:624], h[H_IND], h[H_FUNC] = st, ind, func
            h[H_GLB] = h[H_CLB] = t
            h[H_PROBES] = h[H_RECORDS] = h[H_SNAP] = h[H_MASTER] = h[H_CATHODE] = 0
        h[H_TCNTR] = t
        h[H_NE] = len(share[0])
        h[H_MAXNE] = max(int(h[H_MAXNE]), len(share[0]))
        for s in range(n_spec):
            h[636 + 2 * s + 1] = len(share[1 + s])
            h[636 + 2 * s] = max(int(h[636 + 2 * s]), len(share[1 + s]))
        surf = np.zeros(0)
        diel = _dielectrics(p)
        if r == 0 and diel:
            from . import FIELD_SURFACE_CHARGE
            grid = sim.field(FIELD_SURFACE_CHARGE)
            surf = np.array([grid[j, i] for o in diel for (i, j) in outline_nodes(*o)])
        h[-1] = len(surf)
        ranks.append(Rank(h, surf, share[0], share[1:]))
    if fmt == "posix":
        return write_posix(root, t, ranks)
    return [write_mpiio(mpiio_path(root, t), ranks)]
