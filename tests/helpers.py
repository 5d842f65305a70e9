"""Comparison helpers shared by the parity tests."""

import numpy as np


def f32_bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


def rel_err(got, ref, floor):
    """Elementwise |got-ref| / max(|ref|, floor)."""
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    return np.abs(got - ref) / np.maximum(np.abs(ref), floor)


def kriged_slots(ref_status):
    return np.nonzero(ref_status >= 0)[0]


def neighbour_lists_equal(ref, got, slots_ref, slots_got, cap_ref, cap_got):
    """Neighbour count and index list (first count entries) per slot."""
    rc = ref["nb_count"][slots_ref]
    gc = got["nb_count"][slots_got]
    if not np.array_equal(rc, gc):
        bad = np.nonzero(rc != gc)[0]
        return False, "count differs at %d slots, first slot %d (%d vs %d)" % (
            len(bad), slots_ref[bad[0]], rc[bad[0]], gc[bad[0]])
    cap = min(cap_ref, cap_got)
    ri = ref["nb_index"].reshape(-1, cap_ref)[slots_ref, :cap]
    gi = got["nb_index"].reshape(-1, cap_got)[slots_got, :cap]
    valid = np.arange(cap)[None, :] < rc[:, None]
    diff = (ri != gi) & valid
    if diff.any():
        s = np.nonzero(diff.any(axis=1))[0]
        return False, "index lists differ at %d slots, first slot %d" % (len(s), slots_ref[s[0]])
    return True, ""
