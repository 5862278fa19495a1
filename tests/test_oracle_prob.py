"""The oracle's ProbVoxelMap insert and mergeOccupied against the reference's
own rules and its ProbMap2DistMap example (two overlapping boxes inserted
with maximal occupied / free probability, merged at threshold 0.55)."""
import numpy as np

import oracle
import refgeom


def test_float_to_probability_matches_reference_encoding():
    # ProbabilisticVoxel::floatToProbability: clamp to [0,1], * 254 - 127, truncate to int8
    assert oracle.float_to_probability(0.5) == 0
    assert oracle.float_to_probability(0.55) == 12
    assert oracle.float_to_probability(1.0) == 127
    assert oracle.float_to_probability(0.0) == -127
    assert oracle.float_to_probability(2.0) == 127
    assert oracle.float_to_probability(-1.0) == -127
    assert oracle.float_to_probability(0.25) == -63  # -63.5 truncates toward zero


def test_update_rules():
    dims = (4, 4, 4)
    one = np.array([[1.5, 1.5, 1.5]], np.float32)
    m = oracle.pvm_empty(dims)
    oracle.pvm_insert(m, dims, 1.0, one, 1)  # occupied from unknown: 0 + 72
    i = 1 + 4 * 1 + 16 * 1
    assert m[i] == 72
    oracle.pvm_insert(m, dims, 1.0, one, 1)
    assert m[i] == 127  # saturates
    oracle.pvm_insert(m, dims, 1.0, one, 0)
    assert m[i] == 117  # free: -10
    oracle.pvm_insert(m, dims, 1.0, one, 4)
    assert m[i] == -8  # eBVM_MAX_FREE_PROB: 4 - 129
    oracle.pvm_insert(m, dims, 1.0, one, 3)
    assert m[i] == -128  # eBVM_UNKNOWN resets
    oracle.pvm_insert(m, dims, 1.0, one, 254)
    assert m[i] == 125  # eBVM_MAX_OCC_PROB from unknown
    assert oracle.pvm_insert(m, dims, 1.0, np.array([[9.0, 0.5, 0.5]], np.float32), 1)  # outside flag
    assert (np.delete(m, i) == -128).all()


def test_prob_map_to_distance_map_example():
    dims = (128, 128, 128)
    box1 = refgeom.box_of_points((40, 40, 40), (60, 60, 60), 0.9)
    box2 = refgeom.box_of_points((50, 50, 50), (70, 70, 70), 0.9)
    p = oracle.pvm_empty(dims)
    oracle.pvm_insert(p, dims, 1.0, box1, 254)  # eBVM_MAX_OCC_PROB
    oracle.pvm_insert(p, dims, 1.0, box2, 4)    # eBVM_MAX_FREE_PROB
    d = oracle.dvm_empty(dims)
    oracle.dvm_merge_occupied(d, p, dims, (0, 0, 0), 0.55)
    sites = d != 0x3FFFFFFF
    # the box generator stops below 60 (step 0.9 from 40): voxels 40..59 of box 1
    # minus the overlap 50..59 with box 2
    assert int(sites.sum()) == 20 ** 3 - 10 ** 3
    z, y, x = np.unravel_index(np.nonzero(sites)[0], (128, 128, 128))
    assert x.min() == 40 and x.max() == 59
    v = d[sites]
    assert np.array_equal(v & 0x3FF, x) and np.array_equal((v >> 10) & 0x3FF, y) and np.array_equal(v >> 20, z)
    # an offset shifts the stored sites, not the voxels written
    d2 = oracle.dvm_empty(dims)
    oracle.dvm_merge_occupied(d2, p, dims, (1, 2, 3), 0.55)
    assert np.array_equal(d2 != 0x3FFFFFFF, sites)
    assert np.array_equal(d2[sites], d[sites] + 1 + (2 << 10) + (3 << 20))
    oracle.pba(d, dims)
    assert (d != 0x3FFFFFFF).all()
