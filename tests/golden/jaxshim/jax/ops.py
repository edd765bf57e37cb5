"""``jax.ops`` stand-in; golden-vector generation only."""
import numpy as _np
from .numpy import _wrap


def segment_sum(data, segment_ids, num_segments=None, **_k):
    data = _np.asarray(data)
    ids = _np.asarray(segment_ids)
    n = int(num_segments) if num_segments is not None else int(ids.max()) + 1
    out = _np.zeros((n,) + data.shape[1:], dtype=data.dtype)
    _np.add.at(out, ids, data)
    return _wrap(out)
