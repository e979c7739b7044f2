"""The whole path against the reference's own partitioner and against an
independent FP64 eigensolver.

Edge cuts.  The reference's heavy-edge coarsening is not reproducible from a
seed (its permutation and tie-breaks), and this path makes those choices with
a seeded hash, so one seed does not give the same partition on both sides.
Their cut distributions are compared instead: ten seeds of this path on the
GPU against ten seeds of the reference's sgp_partition_graph
(cmg/sgpar.h:2432-2661, its serial build compiled from the reference sources
into oracle/_ref by oracle/Makefile) on the 256 x 256 grid with coarsening
cutoff 32, R-MAT scale 16 and a 3D random geometric graph.  The medians must
agree within 15% (measured: 0.93, 1.01 and 0.98 of the reference's) and the
ranges must overlap.

Fiedler value.  SciPy's FP64 eigensolvers give lambda_2 of the same graphs
(shift-invert Lanczos for the grid and the geometric graph, LOBPCG against
the constant vector for R-MAT).  The path's finest Rayleigh quotient and its
residual ||L x - lambda x|| / (2 max_i d_i) are recomputed on the CPU from
the eigenvector the device returns.  The reference's stopping rule
(|d dot| <= 1e-10, eigensolve_kokkos.h:153) ends the grid and geometric graphs
within 5% of lambda_2.  On R-MAT it ends far above lambda_2 (about 13x on
scale 16), because the shift gb = 2 max d makes the dot change too slowly to
measure progress; the reference does the same.  There the test checks the
bound lambda >= lambda_2 that every vector orthogonal to the constant vector
satisfies.
"""
import numpy as np
import pytest

from ipdps_2021_graph_coarsening_b200 import _lib as L
from ipdps_2021_graph_coarsening_b200 import api
from ipdps_2021_graph_coarsening_b200 import graphs as G
from oracle import bindings as O

pytestmark = pytest.mark.gpu

sp = pytest.importorskip("scipy.sparse")
sla = pytest.importorskip("scipy.sparse.linalg")

CASES = {
    "grid256_c32": (lambda: G.grid2d(256, 256), 32),
    "rmat16": (lambda: G.rmat(16, seed=1), 50),
    "rgg20k": (lambda: G.rgg3d(20000, seed=3), 50),
}
SEEDS = range(100, 110)


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    f, cutoff = CASES[request.param]
    return request.param, f(), cutoff


def test_cut_distribution_matches_reference(partitioner, case):
    name, g, cutoff = case
    if not O.ref_available("serial", cutoff):
        pytest.skip("the reference build (oracle/_ref) is not present")
    ours = [partitioner.partition(g, cutoff=cutoff, rng_state=s).edgecut for s in SEEDS]
    ref = [O.ref_partition_graph(g.row_ptr, g.col, rng_state=s, kind="serial", cutoff=cutoff)[1] for s in SEEDS]
    mo, mr = float(np.median(ours)), float(np.median(ref))
    print(f"{name}: ours median {mo} {sorted(ours)}; reference median {mr} {sorted(ref)}")
    assert abs(mo - mr) <= 0.15 * mr
    assert min(ours) <= max(ref) and min(ref) <= max(ours)


def test_match_cut_distribution_matches_reference(partitioner, case):
    """The heavy-edge matching coarsener with the coarsening-ratio stop
    (options.coarsener = MATCH | RATIO_STOP, the serial driver's
    coarsening_alg bit 0) against the reference's serial matching path
    (sgp_coarsen_heavy_edge_matching, cmg/sgpar.h:364-452, chosen by
    coarsening_alg = 5 at sgpar.h:1356-1365, with its ratio stop at
    :2470-2475): ten seeds each, medians within 15% (measured: 1.11, 0.98 and
    0.98 of the reference's).  The ranges are not required to overlap: on
    R-MAT 16 both spreads are under 1% and this path's cuts sit 1.6% below
    the reference's (425,467..429,775 against 432,756..435,919)."""
    name, g, cutoff = case
    if not O.ref_available("serial", cutoff):
        pytest.skip("the reference build (oracle/_ref) is not present")
    co = L.COARSEN_MATCH | L.COARSEN_RATIO_STOP
    ours = [partitioner.partition(g, cutoff=cutoff, rng_state=s, coarsener=co).edgecut for s in SEEDS]
    ref = [O.ref_partition_graph(g.row_ptr, g.col, rng_state=s, kind="serial", cutoff=cutoff, coarsening_alg=5)[1]
           for s in SEEDS]
    mo, mr = float(np.median(ours)), float(np.median(ref))
    print(f"{name}: matching, ours median {mo} {sorted(ours)}; reference median {mr} {sorted(ref)}")
    assert abs(mo - mr) <= 0.15 * mr


def laplacian(g):
    rows = np.repeat(np.arange(g.n), np.diff(g.row_ptr).astype(np.int64))
    A = sp.csr_matrix((np.ones(len(g.col)), (rows, g.col.astype(np.int64))), shape=(g.n, g.n))
    d = np.asarray(A.sum(axis=1)).ravel()
    return (sp.diags(d) - A).tocsr(), d


def lambda2(name, L, d):
    if name.startswith("rmat"):
        rng = np.random.default_rng(0)
        vals, _ = sla.lobpcg(L, rng.standard_normal((L.shape[0], 4)), M=sp.diags(1.0 / d),
                             Y=np.ones((L.shape[0], 1)), largest=False, tol=1e-9, maxiter=3000)
        return float(np.min(vals))
    vals = sla.eigsh(L.tocsc(), k=2, sigma=-1e-3, which="LM", return_eigenvectors=False)
    return float(np.sort(vals)[1])


def test_fiedler_value_against_fp64_eigensolver(partitioner, case):
    name, g, cutoff = case
    L, d = laplacian(g)
    lam2 = lambda2(name, L, d)
    if name.startswith("grid"):
        assert abs(lam2 - (2 - 2 * np.cos(np.pi / 256))) <= 1e-9 * lam2   # closed form
    seed = 7
    r = partitioner.partition(g, cutoff=cutoff, rng_state=seed)
    # the same partition's eigenvector through the lower boundary: coarsening
    # advances the rng, the eigensolve continues from it
    rng = api.PCG32(state=seed, inc=1)
    h = partitioner.generate_coarse_graphs(g, cutoff=cutoff, rng=rng)
    try:
        x = h.eigensolve(rng=rng)
    finally:
        h.free()
    # the device's Rayleigh quotient and residual, recomputed on the CPU
    Lx = L @ x
    lam = float(x @ Lx / (x @ x))
    res = float(np.linalg.norm(Lx - lam * x) / np.linalg.norm(x) / (2 * d.max()))
    assert abs(lam - r.lam) <= 1e-9 * lam
    assert abs(res - r.residual) <= 1e-6 * res + 1e-15
    rel = (lam - lam2) / lam2
    print(f"{name}: lambda {lam:.9e} lambda_2 {lam2:.9e} rel {rel:.3e} residual {res:.3e}")
    assert lam >= lam2 * (1 - 1e-9)
    if not name.startswith("rmat"):
        assert rel <= 0.05



def test_residual_with_hub_rows(partitioner):
    """The reported eigenvalue and residual on a graph whose finest level has
    rows of more than 8192 entries (R-MAT 18: 19 such hubs, up to 25k
    entries), which the residual pass gives a block each: both recomputed on
    the CPU from the eigenvector."""
    g = G.rmat(18, seed=2)
    L, d = laplacian(g)
    assert d.max() > 8192
    seed = 11
    r = partitioner.partition(g, rng_state=seed)
    rng = api.PCG32(state=seed, inc=1)
    h = partitioner.generate_coarse_graphs(g, rng=rng)
    try:
        x = h.eigensolve(rng=rng)
    finally:
        h.free()
    Lx = L @ x
    lam = float(x @ Lx / (x @ x))
    res = float(np.linalg.norm(Lx - lam * x) / np.linalg.norm(x) / (2 * d.max()))
    assert abs(lam - r.lam) <= 1e-9 * lam
    assert abs(res - r.residual) <= 1e-6 * res + 1e-15
