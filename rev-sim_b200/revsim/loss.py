"""Loss specifications: the reference's RDF loss and the fixed-grid L2 RDF loss.

Reference loss (water.jl:616-713): L1 distance between the smoothed O-O and O-H RDFs
on the grid 0.1:0.0005:2.5 nm (width 0.0005, window 0.04 nm) and the Soper 2013
experimental curves, sampled every 6th grid point (O-O indices 323:6:1805, O-H
125:6:1805, 1-based).  ``read_rdf_data`` parses the reference's data file when a
caller supplies its path.
"""

import numpy as np

from .engine import RdfTerm

REF_X_MIN, REF_STEP, REF_N_GRID = 0.1, 0.0005, 4801   # Int(cld(2.5 - 0.1, 0.0005)) + 1
REF_WIDTH, REF_CUTOFF = 0.0005, 0.04


def read_rdf_data(path):
    """water.jl:616-629: skip two header rows; O-O rows 87:334, O-H 54:334, H-H 74:334
    (1-based, after the skip) of columns 2, 4 and 6."""
    oo, oh, hh = [], [], []
    with open(path) as f:
        lines = f.read().splitlines()[2:]
    for line in lines:
        cols = line.split()
        if len(cols) < 6:
            continue
        oo.append(float(cols[1]))
        oh.append(float(cols[3]))
        hh.append(float(cols[5]))
    return np.array(oo[86:334]), np.array(oh[53:334]), np.array(hh[73:334])


def reference_rdf_terms(target_oo, target_oh, weight=1.0):
    """The two L1 terms of loss_rdf (water.jl:702-713) against the given targets
    (248 O-O values, 281 O-H values)."""
    target_oo = np.asarray(target_oo, dtype=np.float64)
    target_oh = np.asarray(target_oh, dtype=np.float64)
    return [
        RdfTerm(0, 0, REF_X_MIN, REF_STEP, REF_WIDTH, REF_CUTOFF, REF_N_GRID, 322, 6, target_oo,
                1, weight),
        RdfTerm(0, 1, REF_X_MIN, REF_STEP, REF_WIDTH, REF_CUTOFF, REF_N_GRID, 124, 6, target_oh,
                1, weight),
    ]


def oo_l2_term(target, n_bins=200, r_max=1.0, width=0.0005, exp_cutoff=0.04, weight=1.0):
    """Squared error of the smoothed O-O RDF on n_bins grid points step, 2 step, ..., r_max."""
    step = r_max / n_bins
    target = np.asarray(target, dtype=np.float64)
    return RdfTerm(0, 0, step, step, width, exp_cutoff, n_bins, 0, 1, target, 2, weight)
