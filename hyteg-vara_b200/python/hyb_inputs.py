"""Synthetic inputs of the benchmark configurations (no dataset is involved).

Every input is keyed by geometry, not by memory layout, so the GPU path and the CPU
oracle see identical values:
  * right-hand side f ~ U[-1, 1] i.i.d. per micro-vertex, a SplitMix64 hash of
    (seed, the vertex's integer position on the global lattice of spacing 1/lattice);
  * coefficient k = exp(g), g a stationary Gaussian random field with squared-
    exponential covariance (correlation length, sigma), drawn by random Fourier
    features from a seeded generator;
  * meshes: the reference's cuboid generator (MeshInfo::meshCuboid,
    src/hyteg/mesh/MeshGenCuboid.cpp:34-160) restated.
"""
import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def mesh_cuboid(nx, ny, nz, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    """Vertices x-fastest, six tets per cube from the hexahedron node table, cells in the
    lexicographic order of their vertex-id lists (the order the reference numbers them)."""
    hx, hy, hz = [(hi[d] - lo[d]) / n for d, n in enumerate((nx, ny, nz))]
    coords = []
    for iz in range(nz + 1):
        for iy in range(ny + 1):
            for ix in range(nx + 1):
                coords.append((lo[0] + ix * hx, lo[1] + iy * hy, lo[2] + iz * hz))
    tnode = [(4, 5, 7, 3), (0, 3, 1, 4), (4, 1, 5, 3), (5, 6, 7, 2), (1, 3, 2, 5), (7, 2, 3, 5)]
    off = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]

    def vid(i, j, k):
        return k * (nx + 1) * (ny + 1) + j * (nx + 1) + i

    tets = set()
    for iz in range(nz):
        for iy in range(ny):
            for ix in range(nx):
                for t in tnode:
                    tets.add(tuple(vid(ix + off[m][0], iy + off[m][1], iz + off[m][2]) for m in t))
    return np.array(coords, np.float64), np.array(sorted(tets), np.int64)


def splitmix64(x):
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & _M64
    z = x
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
    return z ^ (z >> np.uint64(31))


def uniform_rhs(xyz, seed, lattice):
    key = np.rint(np.asarray(xyz) * lattice).astype(np.int64)
    k = (key[:, 0].astype(np.uint64) * np.uint64(1_000_003) + key[:, 1].astype(np.uint64)) * np.uint64(1_000_033) \
        + key[:, 2].astype(np.uint64)
    with np.errstate(over="ignore"):
        h = splitmix64(k ^ (np.uint64(seed) * np.uint64(0xD1B54A32D192ED03)))
    return (h >> np.uint64(11)).astype(np.float64) / float(1 << 53) * 2.0 - 1.0


def grf_features(corr_len=0.2, seed=1, modes=64):
    """Random Fourier features (wave vectors ~ N(0, 1/corr_len^2), phases ~ U[0, 2 pi)) of a
    Gaussian random field with a squared-exponential covariance of length corr_len."""
    rng = np.random.default_rng(seed)
    w = rng.normal(0.0, 1.0 / corr_len, size=(modes, 3))
    ph = rng.uniform(0.0, 2.0 * np.pi, size=modes)
    return w, ph


def grf_coefficient(xyz, corr_len=0.2, sigma=1.0, seed=1, modes=64):
    w, ph = grf_features(corr_len, seed, modes)
    g = sigma * np.sqrt(2.0 / modes) * np.cos(np.asarray(xyz) @ w.T + ph).sum(axis=1)
    return np.exp(g)


def shell_coefficient(xyz, radial=5.0, sigma=0.5, seed=2, corr_len=0.2, modes=64):
    """k = exp(radial (1 - r)) times lognormal noise exp(sigma g), g a Gaussian random field
    (random Fourier features of correlation length corr_len)."""
    w, ph = grf_features(corr_len, seed, modes)
    x = np.asarray(xyz)
    r = np.sqrt((x * x).sum(axis=1))
    g = sigma * np.sqrt(2.0 / modes) * np.cos(x @ w.T + ph).sum(axis=1)
    return np.exp(radial * (1.0 - r) + g)
