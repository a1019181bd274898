"""``jax.ops.segment_sum`` (test infrastructure)."""

import numpy as np

from .numpy import _wrap


def segment_sum(data, segment_ids, num_segments=None):
    data = np.asarray(data)
    ids = np.asarray(segment_ids)
    n = int(num_segments) if num_segments is not None else int(ids.max()) + 1
    out = np.zeros((n,) + data.shape[1:], dtype=data.dtype)
    np.add.at(out, ids, data)
    return _wrap(out)
