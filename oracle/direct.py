"""Oracle restatement of the dense debug path ``bndiag_of_inv_direct!``
(src/matinvertndiag_direct.jl:17-61) and its copying form (:78-85).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

The reference densifies M (``Array(M)``, :21), inverts it with the backend's
``be_inv`` (LAPACK getrf + getri through ``inv``, src/backend_cpu.jl:143-145;
numpy's ``inv`` is the same LAPACK pair), and writes the blocks of the out
band of the inverse into M itself (:32-58): stored entries of M outside the
band stay as they are.
"""

import numpy as np


def bndiag_of_inv_direct(M, block_sizes, ndiag):
    """Returns (dense result, inverse): the dense form of the matrix the
    reference returns, and the whole inverse."""
    D = np.asarray(M.toarray() if hasattr(M, "toarray") else M, dtype=np.complex128)
    inv = np.linalg.inv(D)
    out = D.copy()
    off = np.concatenate([[0], np.cumsum(block_sizes)])
    w = (ndiag["out"] - 1) // 2
    npl = len(block_sizes)
    for ix in range(npl):
        for jx in range(max(0, ix - w), min(npl, ix + w + 1)):
            out[off[ix]:off[ix + 1], off[jx]:off[jx + 1]] = inv[off[ix]:off[ix + 1], off[jx]:off[jx + 1]]
    return out, inv
