"""Host planner (product) bit-exact against the reference's compiled plans."""
import numpy as np
import pytest

from dcs245_classical_sampling_b200 import plan as P
from dcs245_classical_sampling_b200.workloads import build_workload, WORKLOADS


@pytest.mark.parametrize("name", ["c1", "small", "c2", "c64plan"])
def test_block_plan_matches_reference(golden, name):
    case, arrays = golden(name)
    bp = P.build_block_plan(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                            case["parity_operations"], case["open_vertices"])
    ref = case["plan"]
    assert bp.order == ref["order"]
    assert sorted(bp.fixed) == ref["fixed"]
    assert bp.fut == ref["fut"]
    assert bp.stop == ref["stop"]
    assert bp.rmax == ref["rmax"] and bp.work == ref["work"]
    assert bp.maxslots == ref["maxslots"] and bp.inplace_rmax == ref["inplace_rmax"]
    assert list(bp.terminal_slots) == ref["terminal_slots"]
    assert bp.terminal_basis == ref["terminal_basis"]
    assert [list(e) for e in bp.open_edges] == ref["open_edges"]
    for mine, theirs in zip(bp.steps, ref["steps"]):
        assert (mine.v, mine.j, mine.kind, mine.beta, mine.K, mine.Ka, mine.pivot, mine.pivot_a, mine.free) == \
            (theirs["v"], theirs["j"], theirs["kind"], theirs["beta"], theirs["K"], theirs["Ka"],
             theirs["pivot"], theirs["pivot_a"], theirs["free"])
        assert list(mine.active_in) == theirs["active_in"] and list(mine.active_out) == theirs["active_out"]


def test_cut_ranks_and_chooser_match_reference(golden):
    c, _ = golden("chooser")
    from dcs245_classical_sampling_b200.circuits import build_ring_instance
    inst = build_ring_instance(c["n"], c["depth"], c["t_count"], c["seed"])
    A = inst["graph"]
    assert list(P.prefix_cut_ranks(A, c["order"])) == c["cut_ranks"]
    edges = [(int(a), int(b)) for a, b in zip(*np.nonzero(np.triu(A, 1)))]
    ops, S = P.choose_parity_slices(len(A), edges, c["order"], 3, seed=0)
    assert [list(o) for o in ops] == c["ops"] and S == c["removed"]


def test_reference_errors():
    from dcs245_classical_sampling_b200.circuits import build_ring_instance
    inst = build_ring_instance(4, 3, 2, 1)
    args = (inst["graph"], inst["unitaries"], 4, list(inst["order"]))
    with pytest.raises(ValueError):
        P.build_block_plan(*args, [], [1, 1])            # repeated free vertex
    with pytest.raises(ValueError):
        P.build_block_plan(*args, [], [5])               # not a data vertex
    with pytest.raises(ValueError):
        P.build_block_plan(*args, [("Z", 0, None)], [1])  # slicing a data vertex
    with pytest.raises(ValueError):
        P.build_block_plan(*args, [("Q", 4, None)], [1])  # unknown parity kind


def test_workload_cache_is_reproducible():
    for name in ["ring16_d20_t24_k8", "ring24_d24_t60_k10"]:
        cached = build_workload(name)
        fresh = build_workload(name, use_cache=False)
        assert cached["parity_operations"] == fresh["parity_operations"]


def test_workload_sizes():
    for name, (n, depth, t, seed, k, npar) in WORKLOADS.items():
        w = build_workload(name)
        assert w["N"] == n + t and len(w["open_vertices"]) == k and len(w["parity_operations"]) == npar


def test_half_storage_argument_errors(golden):
    """alloc rejects the half-storage tier with complex128, with the fused executor, and unknown
    storage names, before touching a device."""
    case, arrays = golden("c1")
    from dcs245_classical_sampling_b200.engine import InplaceConditionalBlockGPU
    eng = InplaceConditionalBlockGPU(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                                     case["parity_operations"], case["open_vertices"])
    for kw in ({"dtype": np.complex128, "storage": "float16"}, {"mode": "fused", "storage": "float16"},
               {"storage": "bfloat16"}):
        with pytest.raises(ValueError):
            eng.alloc(**kw)


def test_native_cut_ranks_equal_gf2_rank_of_each_cut():
    """dcs_prefix_cut_ranks against a plain GF(2) rank of A[prefix, suffix] on random graphs,
    including orders over a subset of the vertices (the chooser's `alive` lists)."""
    rng = np.random.default_rng(11)

    def gf2_rank(M):
        M = M.copy() % 2
        r = 0
        for c in range(M.shape[1]):
            p = [i for i in range(r, M.shape[0]) if M[i, c]]
            if not p:
                continue
            M[[r, p[0]]] = M[[p[0], r]]
            for i in range(M.shape[0]):
                if i != r and M[i, c]:
                    M[i] ^= M[r]
            r += 1
        return r

    for n, dens in ((5, 0.5), (17, 0.3), (70, 0.1), (130, 0.05)):
        A = (rng.random((n, n)) < dens).astype(np.uint8)
        A = np.triu(A, 1)
        A = A | A.T
        for sub in (n, max(2, n - 3)):
            order = [int(v) for v in rng.permutation(n)[:sub]]
            got = P.prefix_cut_ranks(A, order)
            want = [gf2_rank(A[np.ix_(order[:i], order[i:])]) for i in range(1, sub)]
            assert list(got) == want
    with pytest.raises(Exception):
        P.prefix_cut_ranks(np.zeros((3, 3), np.uint8), [0, 1, 5])


@pytest.mark.parametrize("name", ["c1", "small", "c2"])
def test_gather_plan_matches_reference(golden, name):
    """The gather form of the plan (the reference's ConditionalBlockGPU, scan_plan.make_plan):
    every step's ranks, sign functional, right inverse and kernel, the rank profile, rmax, work
    and the terminal basis, bit for bit."""
    from dcs245_classical_sampling_b200.plan import build_block_plan, build_gather_plan
    case, arrays = golden(name)
    g = golden("gather")[0][name]
    bp = build_block_plan(arrays["graph"], arrays["unitaries"], case["n"], case["order"],
                          case["parity_operations"], case["open_vertices"])
    gp = build_gather_plan(bp)
    assert gp.rmax == g["rmax"] and gp.work == g["work"] and bp.stop == g["stop"]
    assert gp.terminal_basis == g["terminal_basis"]
    assert gp.rank_profile == g["rank_profile"]
    assert len(gp.steps) == len(g["steps"])
    for mine, theirs in zip(gp.steps, g["steps"]):
        for key in ("v", "free", "r_in", "r_out", "beta", "Lcols", "kernel"):
            assert getattr(mine, key) == theirs[key], key
    # the reference's gather blocks equal its in-place blocks (the golden blocks) to rounding
    assert max(g["blocks_rel_l2_vs_inplace"]) < 1e-14
