"""Seeded synthetic block-stencil systems (host side, numpy).

Every workload of the solve path is generated here, once, on the host and fed
identically to the CPU oracle, to the reference build and to the GPU:

* ``grid_system(dims, bs, seed, skew=c)`` — the 2D 5-point / 3D 7-point block
  stencil.  Every grid edge (p, q), p < q, draws ``G`` (bs x bs, iid N(0,1)) and
  adds ``K = G G^T + 0.1 I`` to A_pp and A_qq and ``-K`` to A_pq and A_qp.  Each
  diagonal block then gets ``+0.01 I`` so A is SPD.  With ``skew = c > 0`` each
  edge also draws ``S`` and adds ``c (S - S^T)`` to *both* A_pq and A_qp: since
  ``(S - S^T)^T = -(S - S^T)`` that term is skew-symmetric as a whole, so A is
  nonsymmetric while its symmetric part stays the SPD matrix above.
* ``batch_specs(seed, count)`` — the uneven-size batch of 2D systems.
* ``convection_diffusion_system(...)`` — the 3D convection-diffusion family
  used to train and evaluate the learned preconditioner.
* ``complex_system(dims, bs, seed)`` — a complex (std::complex<double>) block
  system: a grid system plus i times a second one of the same pattern.

Randomness: one Philox4x64-10 stream per system, keyed by the seed
(``numpy.random.Philox(key=seed)``, counter from 0), read as uniform doubles
``(u64 >> 11) * 2^-53``; normals come from this module's own Box-Muller
transform, not from a library sampler whose algorithm could change.  Draw order:
all G (x-edges, then y-edges, then z-edges, each in increasing p), then all S,
then b.

Node numbering is lexicographic, ``idx = i + nx*j (+ nx*ny*k)``; inside a block
row the columns are stored in increasing order.
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass
from pathlib import Path

import numpy as np


@dataclass
class BSRSystem:
    """A block CSR matrix (row-major bs x bs blocks) and right-hand side(s)."""

    n: int                 # block rows (= block columns)
    bs: int                # block size
    row_ptr: np.ndarray    # int32 [n+1]
    col_idx: np.ndarray    # int32 [nnzb]
    vals: np.ndarray       # float64 [nnzb, bs, bs]
    b: np.ndarray          # float64 [n * bs * nrhs]
    nrhs: int = 1
    name: str = ""

    @property
    def nnzb(self) -> int:
        return int(self.col_idx.shape[0])

    def to_dense(self) -> np.ndarray:
        n, bs = self.n, self.bs
        A = np.zeros((n * bs, n * bs))
        for i in range(n):
            for t in range(self.row_ptr[i], self.row_ptr[i + 1]):
                j = self.col_idx[t]
                A[i * bs:(i + 1) * bs, j * bs:(j + 1) * bs] = self.vals[t]
        return A


def rng_for(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(key=np.uint64(seed)))


def normals(rng: np.random.Generator, count: int) -> np.ndarray:
    """``count`` N(0,1) draws by Box-Muller: u1 block then u2 block."""
    m = (count + 1) // 2
    u1 = rng.random(m)
    u2 = rng.random(m)
    r = np.sqrt(-2.0 * np.log1p(-u1))
    th = 2.0 * math.pi * u2
    z = np.empty(2 * m)
    z[0::2] = r * np.cos(th)
    z[1::2] = r * np.sin(th)
    return z[:count]


def _stencil_layout(dims: tuple[int, ...]):
    """Slot order (ascending column) and per-slot (axis, sign) for a grid."""
    nd = len(dims)
    # slots: -axis for axis nd-1..0, self, +axis for axis 0..nd-1
    slots = [(ax, -1) for ax in reversed(range(nd))] + [(None, 0)] + [(ax, +1) for ax in range(nd)]
    strides = [1]
    for d in dims[:-1]:
        strides.append(strides[-1] * d)
    return slots, strides


def assemble_grid(dims: tuple[int, ...], bs: int, edge_blocks: list[tuple[np.ndarray, np.ndarray]],
                  diag: np.ndarray):
    """Assemble a BSR stencil matrix.

    edge_blocks[ax] = (B_plus, B_minus): blocks for slot +ax of row p and slot
    -ax of row q = p + stride[ax], each shaped like the edge array of that axis
    (grid shape with axis length reduced by one, C-order over reversed dims).
    diag: (n, bs, bs) diagonal blocks.
    """
    nd = len(dims)
    n = int(np.prod(dims))
    slots, strides = _stencil_layout(dims)
    shape = tuple(reversed(dims))  # C-order array index [k, j, i]
    coords = np.indices(shape).reshape(nd, -1)[::-1]  # coords[ax] over nodes in idx order
    idx = np.arange(n, dtype=np.int64)
    mask = np.zeros((n, len(slots)), dtype=bool)
    cols = np.zeros((n, len(slots)), dtype=np.int64)
    for s, (ax, sg) in enumerate(slots):
        if ax is None:
            mask[:, s] = True
            cols[:, s] = idx
        elif sg < 0:
            mask[:, s] = coords[ax] > 0
            cols[:, s] = idx - strides[ax]
        else:
            mask[:, s] = coords[ax] < dims[ax] - 1
            cols[:, s] = idx + strides[ax]
    counts = mask.sum(1)
    row_ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    nnzb = int(row_ptr[-1])
    pos = row_ptr[:-1, None] + np.cumsum(mask, axis=1) - 1
    col_idx = np.empty(nnzb, dtype=np.int32)
    col_idx[pos[mask]] = cols[mask]
    vals = np.empty((nnzb, bs, bs))
    self_slot = nd
    vals[pos[:, self_slot]] = diag
    grid_pos = pos.reshape(*shape, len(slots))
    for ax in range(nd):
        sl_p = [slice(None)] * nd
        sl_m = [slice(None)] * nd
        arr_ax = nd - 1 - ax  # array axis of grid axis ax
        sl_p[arr_ax] = slice(0, shape[arr_ax] - 1)
        sl_m[arr_ax] = slice(1, shape[arr_ax])
        s_plus = slots.index((ax, +1))
        s_minus = slots.index((ax, -1))
        bp, bm = edge_blocks[ax]
        vals[grid_pos[tuple(sl_p) + (s_plus,)].ravel()] = bp.reshape(-1, bs, bs)
        vals[grid_pos[tuple(sl_m) + (s_minus,)].ravel()] = bm.reshape(-1, bs, bs)
    return row_ptr.astype(np.int32), col_idx, vals


def grid_system(dims: tuple[int, ...], bs: int, seed: int, skew: float = 0.0, nrhs: int = 1,
                k_shift: float = 0.1, diag_shift: float = 0.01, name: str = "") -> BSRSystem:
    """The block stencil system described in the module docstring."""
    dims = tuple(int(d) for d in dims)
    nd = len(dims)
    n = int(np.prod(dims))
    shape = tuple(reversed(dims))
    rng = rng_for(seed)
    eye = np.eye(bs)
    edge_shapes = []
    for ax in range(nd):
        es = list(shape)
        es[nd - 1 - ax] -= 1
        edge_shapes.append(tuple(es))
    n_edges = [int(np.prod(s)) for s in edge_shapes]
    Ks = []
    for ax in range(nd):
        G = normals(rng, n_edges[ax] * bs * bs).reshape(n_edges[ax], bs, bs)
        K = G @ G.transpose(0, 2, 1)
        K += k_shift * eye
        Ks.append(K)
    Ws = [None] * nd
    if skew != 0.0:
        for ax in range(nd):
            S = normals(rng, n_edges[ax] * bs * bs).reshape(n_edges[ax], bs, bs)
            Ws[ax] = skew * (S - S.transpose(0, 2, 1))
    b = 2.0 * rng.random(n * bs * nrhs) - 1.0
    diag = np.zeros(shape + (bs, bs))
    edge_blocks = []
    for ax in range(nd):
        K = Ks[ax].reshape(edge_shapes[ax] + (bs, bs))
        arr_ax = nd - 1 - ax
        lo = [slice(None)] * nd
        hi = [slice(None)] * nd
        lo[arr_ax] = slice(0, shape[arr_ax] - 1)
        hi[arr_ax] = slice(1, shape[arr_ax])
        diag[tuple(lo)] += K
        diag[tuple(hi)] += K
        off = -Ks[ax]
        if Ws[ax] is not None:
            off = off + Ws[ax]
        edge_blocks.append((off, off))
    diag = diag.reshape(n, bs, bs)
    diag += diag_shift * eye
    row_ptr, col_idx, vals = assemble_grid(dims, bs, edge_blocks, diag)
    return BSRSystem(n=n, bs=bs, row_ptr=row_ptr, col_idx=col_idx, vals=vals, b=b, nrhs=nrhs,
                     name=name or f"grid{'x'.join(map(str, dims))}_bs{bs}_s{seed}")


def gaussian_field(rng: np.random.Generator, dims: tuple[int, ...], corr_len: float) -> np.ndarray:
    """Stationary Gaussian random field on the cells, unit variance, covariance
    ``exp(-r^2 / (2 corr_len^2))``: white noise (this module's normals, in idx
    order) convolved with a separable Gaussian kernel of std ``corr_len/sqrt(2)``
    (periodic wrap, taps to 3 std, each axis' taps scaled to unit L2 norm).
    Returned in idx order (length prod(dims))."""
    shape = tuple(reversed(dims))
    w = normals(rng, int(np.prod(dims))).reshape(shape)
    s = corr_len / math.sqrt(2.0)
    rad = int(math.ceil(3.0 * s))
    t = np.arange(-rad, rad + 1)
    k = np.exp(-(t * t) / (2.0 * s * s))
    k /= math.sqrt(float(np.sum(k * k)))
    for a in range(len(shape)):
        acc = np.zeros_like(w)
        for tap, kt in zip(t, k):
            acc += kt * np.roll(w, int(tap), axis=a)
        w = acc
    return w.reshape(-1)


def complex_system(dims: tuple[int, ...], bs: int, seed: int, skew: float = 0.3, imag: float = 0.3,
                   name: str = "") -> BSRSystem:
    """A complex block system (T = std::complex<double>): the real block stencil
    system of ``grid_system(dims, bs, seed, skew)`` plus i * imag times a second
    one of the same pattern (seed + 7919), and the right-hand side
    b + i * b'.  vals is complex128 [nnzb, bs, bs]; b is complex128 [n * bs]."""
    re = grid_system(dims, bs, seed, skew=skew)
    im = grid_system(dims, bs, seed + 7919, skew=skew)
    vals = re.vals + 1j * imag * im.vals
    b = re.b + 1j * im.b
    return BSRSystem(n=re.n, bs=bs, row_ptr=re.row_ptr, col_idx=re.col_idx, vals=vals, b=b,
                     name=name or f"complex_{len(dims)}d_bs{bs}_s{seed}")


def complex_embedding(vals: np.ndarray) -> np.ndarray:
    """The real 2bs x 2bs blocks of complex bs x bs blocks: complex entry
    a = ar + i ai at (r, c) becomes [[ar, -ai], [ai, ar]] at rows 2r, 2r+1 and
    columns 2c, 2c+1, so a complex vector stored as interleaved (re, im)
    doubles is the real vector the embedded blocks act on."""
    v = np.asarray(vals, dtype=np.complex128)
    nb, bs, _ = v.shape
    out = np.empty((nb, bs, 2, bs, 2))
    out[:, :, 0, :, 0] = v.real
    out[:, :, 0, :, 1] = -v.imag
    out[:, :, 1, :, 0] = v.imag
    out[:, :, 1, :, 1] = v.real
    return out.reshape(nb, 2 * bs, 2 * bs)


@dataclass
class ConvDiffSpec:
    """Per-system data of a convection-diffusion block system: cell
    conductivities, the velocity and the block coupling matrix."""

    dims: tuple[int, ...]
    kappa: np.ndarray     # (n,) exp(sigma * field), idx order
    velocity: np.ndarray  # (nd,)
    M: np.ndarray         # (bs, bs) SPD coupling of the bs unknowns of a cell
    b: np.ndarray         # (n * bs * nrhs,)


def convection_diffusion_spec(dims: tuple[int, ...], bs: int, seed: int, sigma: float = 1.0,
                              corr_len: float = 8.0, speed: float = 0.5, nrhs: int = 1) -> ConvDiffSpec:
    """Draws, in order: the field's normals (n), the velocity direction's normals
    (nd), G (bs x bs normals), then b ~ U[-1, 1]."""
    dims = tuple(int(d) for d in dims)
    n = int(np.prod(dims))
    rng = rng_for(seed)
    g = gaussian_field(rng, dims, corr_len)
    kappa = np.exp(sigma * g)
    u = normals(rng, len(dims))
    vel = speed * u / math.sqrt(float(np.sum(u * u)))
    G = normals(rng, bs * bs).reshape(bs, bs)
    M = G @ G.T / bs + 0.1 * np.eye(bs)
    b = 2.0 * rng.random(n * bs * nrhs) - 1.0
    return ConvDiffSpec(dims, kappa, vel, M, b)


def convection_diffusion_system(dims: tuple[int, ...], bs: int, seed: int, sigma: float = 1.0,
                                corr_len: float = 8.0, speed: float = 0.5, diag_shift: float = 0.01,
                                nrhs: int = 1, spec: ConvDiffSpec | None = None) -> BSRSystem:
    """3D (or 2D) convection-diffusion block system with bs unknowns per cell.

    Cell conductivities kappa = exp(sigma * g), g the unit-variance Gaussian
    field above (correlation length corr_len cells); edge (p, q = p + e_ax)
    conductivity is the harmonic mean ``2 kp kq / (kp + kq)``.  Diffusion couples
    the bs unknowns through the SPD block M = G G^T / bs + 0.1 I; convection by
    the constant velocity v (uniform direction, |v| = speed) is first-order
    upwind on each unknown.  Per edge with c = v_ax:
        A_pp += k_e M + max(-c, 0) I,   A_pq = -k_e M - max(-c, 0) I,
        A_qq += k_e M + max(c, 0) I,    A_qp = -k_e M - max(c, 0) I,
    then every diagonal block gets + diag_shift I.
    """
    dims = tuple(int(d) for d in dims)
    sp = spec or convection_diffusion_spec(dims, bs, seed, sigma, corr_len, speed, nrhs)
    nd = len(dims)
    n = int(np.prod(dims))
    shape = tuple(reversed(dims))
    kap = sp.kappa.reshape(shape)
    eye = np.eye(bs)
    diag = np.zeros(shape + (bs, bs))
    edge_blocks = []
    for ax in range(nd):
        arr_ax = nd - 1 - ax
        lo = [slice(None)] * nd
        hi = [slice(None)] * nd
        lo[arr_ax] = slice(0, shape[arr_ax] - 1)
        hi[arr_ax] = slice(1, shape[arr_ax])
        kp, kq = kap[tuple(lo)], kap[tuple(hi)]
        ke = 2.0 * kp * kq / (kp + kq)
        KM = ke[..., None, None] * sp.M
        c = float(sp.velocity[ax])
        cp, cq = max(-c, 0.0), max(c, 0.0)
        diag[tuple(lo)] += KM + cp * eye   # A_pp: edge towards +axis of p
        diag[tuple(hi)] += KM + cq * eye   # A_qq: edge towards -axis of q
        edge_blocks.append((-KM - cp * eye, -KM - cq * eye))
    diag = diag.reshape(n, bs, bs)
    diag += diag_shift * eye
    row_ptr, col_idx, vals = assemble_grid(dims, bs, edge_blocks, diag)
    return BSRSystem(n=n, bs=bs, row_ptr=row_ptr, col_idx=col_idx, vals=vals, b=sp.b.copy(), nrhs=nrhs,
                     name=f"convdiff{'x'.join(map(str, dims))}_bs{bs}_s{seed}")


def random_blocksp(m: int, bs: int, n_col: int, seed: int, n: int | None = None) -> BSRSystem:
    """A random block matrix in the manner of the reference's rand_BlockSp
    (blocksp_utility.hpp:463-490): each block row draws n_col random block
    columns (a repeated column overwrites its block, so rows keep the order of
    first appearance and may hold fewer blocks) with block entries uniform in
    [0, 1).  Seeded Philox draws replace the reference's rand() and
    default_random_engine, whose sequences are implementation-defined."""
    n = m if n is None else n
    rng = rng_for(seed)
    cols = np.minimum((rng.random(m * n_col) * n).astype(np.int64), n - 1).reshape(m, n_col)
    vals = rng.random(m * n_col * bs * bs).reshape(m, n_col, bs, bs)
    rp, ci, vs = [0], [], []
    for i in range(m):
        row = {}
        for t in range(n_col):
            row[int(cols[i, t])] = vals[i, t]
        ci.extend(row.keys())
        vs.extend(row.values())
        rp.append(len(ci))
    return BSRSystem(n=m, bs=bs, row_ptr=np.array(rp, dtype=np.int32), col_idx=np.array(ci, dtype=np.int32),
                     vals=np.array(vs).reshape(-1, bs, bs), b=2.0 * rng.random(m * bs) - 1.0,
                     name=f"rand{m}_bs{bs}_c{n_col}_s{seed}")


# ---- the named workloads ----------------------------------------------------

def config0(seed: int = 0, side: int = 64) -> BSRSystem:
    """2D side^2 cells, 5-point, 4x4 blocks (B=2, D=2), SPD: pCG + block IChol0."""
    return grid_system((side, side), 4, seed, name=f"cfg0_2d{side}_bs4")


def config1(seed: int = 1, side: int = 64) -> BSRSystem:
    """3D side^3, 7-point, 8x8 blocks (B=4, D=2), skew c = 0.3: pGMRES-DR + ILU0."""
    return grid_system((side, side, side), 8, seed, skew=0.3, name=f"cfg1_3d{side}_bs8")


def config2b(seed: int = 2, side: int = 48) -> BSRSystem:
    """3D side^3, 7-point, 16x16 blocks (B=8, D=2), skew c = 0.3."""
    return grid_system((side, side, side), 16, seed, skew=0.3, name=f"cfg2b_3d{side}_bs16")


def batch_specs(seed: int = 3, count: int = 256, lo: int = 32, hi: int = 256):
    """Sides log-uniform in [lo, hi] (side = round(lo * (hi/lo)^u)), bs in {4, 8}."""
    rng = rng_for(seed)
    u = rng.random(count)
    pick = rng.random(count)
    sides = np.rint(lo * (hi / lo) ** u).astype(int)
    bss = np.where(pick < 0.5, 4, 8)
    return [(int(s), int(b), int(seed * 100003 + i)) for i, (s, b) in enumerate(zip(sides, bss))]


def batch_system(side: int, bs: int, seed: int, nrhs: int = 4) -> BSRSystem:
    """One member of the batch: config-0 generator on a side^2 grid, nrhs RHS."""
    return grid_system((side, side), bs, seed, nrhs=nrhs, name=f"batch_2d{side}_bs{bs}_s{seed}")


# ---- binary exchange format used by the CPU reference driver -----------------
# little-endian: magic b"BSPS", int32 version=1, int32 n, int32 bs, int64 nnzb,
# int32 nrhs, then row_ptr (int32 n+1), col_idx (int32 nnzb),
# vals (float64 nnzb*bs*bs), b (float64 n*bs*nrhs).

def write_bsr(path: str | Path, s: BSRSystem) -> None:
    with open(path, "wb") as f:
        f.write(b"BSPS")
        f.write(struct.pack("<iiiqi", 1, s.n, s.bs, s.nnzb, s.nrhs))
        f.write(np.ascontiguousarray(s.row_ptr, dtype="<i4").tobytes())
        f.write(np.ascontiguousarray(s.col_idx, dtype="<i4").tobytes())
        f.write(np.ascontiguousarray(s.vals, dtype="<f8").tobytes())
        f.write(np.ascontiguousarray(s.b, dtype="<f8").tobytes())


def write_complex_bsr(path: str | Path, s: BSRSystem) -> None:
    """The exchange format with magic BSPC: blocks and right-hand side as
    complex (re, im) doubles."""
    with open(path, "wb") as f:
        f.write(b"BSPC")
        f.write(struct.pack("<iiiqi", 1, s.n, s.bs, int(s.row_ptr[-1]), 1))
        f.write(np.ascontiguousarray(s.row_ptr, dtype="<i4").tobytes())
        f.write(np.ascontiguousarray(s.col_idx, dtype="<i4").tobytes())
        f.write(np.ascontiguousarray(s.vals, dtype="<c16").tobytes())
        f.write(np.ascontiguousarray(s.b, dtype="<c16").tobytes())


def read_bsr(path: str | Path) -> BSRSystem:
    raw = Path(path).read_bytes()
    if raw[:4] != b"BSPS":
        raise ValueError("not a BSPS file")
    ver, n, bs, nnzb, nrhs = struct.unpack_from("<iiiqi", raw, 4)
    off = 4 + struct.calcsize("<iiiqi")

    def take(dtype, count):
        nonlocal off
        a = np.frombuffer(raw, dtype=dtype, count=count, offset=off)
        off += a.nbytes
        return a.copy()

    row_ptr = take("<i4", n + 1)
    col_idx = take("<i4", nnzb)
    vals = take("<f8", nnzb * bs * bs).reshape(nnzb, bs, bs)
    b = take("<f8", n * bs * nrhs)
    return BSRSystem(n=n, bs=bs, row_ptr=row_ptr, col_idx=col_idx, vals=vals, b=b, nrhs=nrhs)


def write_vec(path: str | Path, v: np.ndarray) -> None:
    with open(path, "wb") as f:
        f.write(struct.pack("<q", v.size))
        f.write(np.ascontiguousarray(v, dtype="<f8").tobytes())


def read_vec(path: str | Path) -> np.ndarray:
    raw = Path(path).read_bytes()
    (m,) = struct.unpack_from("<q", raw, 0)
    return np.frombuffer(raw, dtype="<f8", count=m, offset=8).copy()
