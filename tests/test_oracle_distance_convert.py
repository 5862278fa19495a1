"""The oracle's distance-field consumers on known cases: one site in an 8^3
map (free-space bytes with and without a robot radius, the flood-fill
initialisation, the distance band -> list conversion)."""
import numpy as np

import oracle


def _one_site():
    d = (8, 8, 8)
    m = oracle.dvm_empty(d)
    oracle.dvm_insert(m, d, 1.0, np.array([[3.5, 3.5, 3.5]], np.float32))
    oracle.pba(m, d)
    return d, m


def test_free_space_bytes():
    d, m = _one_site()
    b = oracle.extract_distances(m, d, 0).reshape(8, 8, 8)  # [z][y][x]
    assert b[3, 3].tolist() == [3, 2, 1, 0, 1, 2, 3, 4]
    assert b[7, 7, 7] == 6  # sqrt(48) = 6.93 -> 6
    r = oracle.extract_distances(m, d, 2).reshape(8, 8, 8)
    # border rule first: x > X - r gives X - x; then x < r gives x
    assert r[3, 3].tolist() == [0, 1, 1, 0, 1, 2, 3, 1]
    empty = oracle.dvm_empty(d)
    assert (oracle.extract_distances(empty, d, 0) == 127).all()


def test_floodfill_init():
    d, m = _one_site()
    b = oracle.extract_distances(m, d, 0)
    f = oracle.init_floodfill(b, 2)
    assert set(np.unique(f).tolist()) == {32765, 32767}
    assert ((b <= 2) == (f == 32765)).all()


def test_distance_band_to_list():
    d, m = _one_site()
    ids, vox = oracle.extract_given_distances(m, d, 1, 1)
    assert len(ids) == 6 + 12 + 8  # squared distances 1, 2 and 3 floor to 1
    assert (np.diff(ids.astype(np.int64)) > 0).all()
    v = vox.reshape(-1, 32)
    assert (v[:, 0] == 0b10010).all() and (v[:, 1:] == 0).all()  # eBVM_OCCUPIED + swept-volume bit 4
    ids0, vox0 = oracle.extract_given_distances(m, d, 0, 0)
    assert ids0.tolist() == [3 + 8 * 3 + 64 * 3] and vox0.reshape(-1, 32)[0, 0] == 0b10
    ids_all, vox_all = oracle.extract_given_distances(m, d, 0, 127)
    assert len(ids_all) == 512
    six = vox_all.reshape(-1, 32)[np.where(ids_all == 7 + 56 + 448)[0][0]]
    assert six[0] == 0b11110010 and six[1] == 0b11 and (six[2:] == 0).all()  # byte 6: bits 4..9
