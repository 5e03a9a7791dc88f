"""Split nodes whose missing bin holds no rows.

best_numeric_missing (cpp/src/histogram.cpp:144-193) tries both missing directions at
every threshold; with an empty missing bin the two gains tie exactly in exact arithmetic,
and the first direction tried (right) wins.  The reference's FP64 histograms of a node
built by subtraction (parent - sibling, histogram.cpp:108-117) keep a rounding residue in
an empty bin whenever the parent was itself derived, and that residue breaks the tie
either way.  The device sums are exact integers, so at such a node the device records
"right" where the reference's direction follows the residue's sign.  No row of the fit
reaches the node with its missing code, so the direction changes neither the fit nor its
predictions on the training rows; the parity tests compare it everywhere else.
"""
import numpy as np


def pair_bin(a, b, n_bins):
    """cpp/include/tidegbm/histogram.hpp:81-85 (uint32 arithmetic)."""
    return ((a.astype(np.uint64) * 2654435761 + b.astype(np.uint64) * 40503) & 0xFFFFFFFF) % n_bins


def _goes_left(tree, k, codes, n_bins):
    """cpp/src/tree.cpp:15-41 for the rows of `codes` (vectorised)."""
    f = int(tree.feature[k])
    ml = bool(tree.missing_left[k])
    st = int(tree.split_type[k]) if hasattr(tree, "split_type") else 0
    a = codes[:, f].astype(np.int64)
    if st == 1:
        b = codes[:, int(tree.feature2[k])].astype(np.int64)
        miss = (a == 0) | (b == 0)
        return np.where(miss, ml, pair_bin(a, b, n_bins) <= int(tree.threshold[k]))
    if st == 2:
        m = np.asarray(tree.cat_left[k], dtype=np.uint64)
        return ((m[a >> 6] >> (a & 63).astype(np.uint64)) & np.uint64(1)).astype(bool)
    return np.where(a == 0, ml, a <= int(tree.threshold[k]))


def empty_missing_nodes(tree, codes, n_bins, rows=None):
    """Axis and pair split nodes of `tree` (a tree of the reference) whose scanned missing
    bin holds none of `rows` (default: all rows of `codes`): code 0 of the split feature
    for an axis split, pair bin 0 for a pair split."""
    codes = np.asarray(codes)
    rows = np.arange(codes.shape[0]) if rows is None else np.asarray(rows)
    out = set()
    stack = [(0, rows)]
    while stack:
        k, r = stack.pop()
        if tree.is_leaf[k]:
            continue
        st = int(tree.split_type[k]) if hasattr(tree, "split_type") else 0
        c = codes[r]
        if st == 0:
            empty = not np.any(c[:, int(tree.feature[k])] == 0)
        elif st == 1:
            z = pair_bin(c[:, int(tree.feature[k])].astype(np.int64), c[:, int(tree.feature2[k])].astype(np.int64),
                         n_bins)
            empty = not np.any(z == 0)
        else:
            empty = False
        if empty:
            out.add(k)
        left = _goes_left(tree, k, c, n_bins)
        stack.append((int(tree.left[k]), r[left]))
        stack.append((int(tree.right[k]), r[~left]))
    return out
