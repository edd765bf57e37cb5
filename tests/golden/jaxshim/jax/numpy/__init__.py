"""``jax.numpy`` stand-in: NumPy functions returning an ndarray subclass that
carries JAX's functional ``.at[...]`` update syntax.  Test infrastructure for
golden-vector generation only."""
import numpy as _np


class JArray(_np.ndarray):
    """ndarray with JAX's ``.at[idx].op(value)`` functional-update property."""

    @property
    def at(self):
        return _At(self)


def _wrap(x):
    if isinstance(x, _np.ndarray) and not isinstance(x, JArray):
        return x.view(JArray)
    if isinstance(x, tuple):
        return type(x)(*[_wrap(v) for v in x]) if hasattr(x, "_fields") else tuple(_wrap(v) for v in x)
    if isinstance(x, list):
        return [_wrap(v) for v in x]
    return x


class _At:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        return _AtOp(self._arr, idx)


def _expand(idx, ndim):
    if not isinstance(idx, tuple):
        idx = (idx,)
    if any(i is Ellipsis for i in idx):
        k = [j for j, i in enumerate(idx) if i is Ellipsis][0]
        nfill = ndim - (len(idx) - 1)
        idx = idx[:k] + (slice(None),) * nfill + idx[k + 1:]
    return idx


class _AtOp:
    def __init__(self, arr, idx):
        self._arr = arr
        self._idx = idx

    def _apply(self, value, op):
        out = _np.array(self._arr, copy=True).view(JArray)
        idx = self._idx
        value = _np.asarray(value)
        if isinstance(idx, _np.ndarray) and idx.dtype == bool:
            pass
        else:
            eidx = _expand(idx, out.ndim)
            arr_pos = [j for j, i in enumerate(eidx)
                       if isinstance(i, _np.ndarray) and i.dtype != bool]
            if arr_pos:
                # JAX drops scatter updates whose integer index is out of bounds.
                assert len(arr_pos) == 1, "shim supports one integer-array index"
                assert all(isinstance(i, slice) for j, i in enumerate(eidx) if j != arr_pos[0]), \
                    "shim supports an integer-array index only together with slices"
                p = arr_pos[0]
                ind = eidx[p]
                dim = out.shape[p]
                valid = (ind >= -dim) & (ind < dim)
                if not valid.all():
                    clipped = _np.clip(ind, -dim, dim - 1)
                    full = eidx[:p] + (clipped,) + eidx[p + 1:]
                    vb = _np.broadcast_to(value, out[full].shape)
                    vb = _np.take(vb, _np.nonzero(valid)[0], axis=p)
                    eidx = eidx[:p] + (ind[valid],) + eidx[p + 1:]
                    value = vb
            idx = eidx
        if op == "set":
            out[idx] = value
        elif op == "add":
            out[idx] = out[idx] + value
        elif op == "multiply":
            out[idx] = out[idx] * value
        elif op == "divide":
            out[idx] = out[idx] / value
        else:
            raise ValueError(op)
        return out

    def set(self, v):
        return self._apply(v, "set")

    def add(self, v):
        return self._apply(v, "add")

    def multiply(self, v):
        return self._apply(v, "multiply")

    def divide(self, v):
        return self._apply(v, "divide")


def _wrapfn(f):
    def g(*a, **k):
        return _wrap(f(*a, **k))
    g.__name__ = getattr(f, "__name__", "fn")
    return g


def argsort(a, axis=-1, **_k):
    return _wrap(_np.argsort(a, axis=axis, kind="stable"))


def reshape(a, shape=None, order="C", newshape=None):
    s = shape if shape is not None else newshape
    return _wrap(_np.reshape(_np.asarray(a), s, order=order))


class _Linalg:
    @staticmethod
    def eigh(a, UPLO=None, symmetrize_input=True):
        a = _np.asarray(a)
        if symmetrize_input:
            a = 0.5 * (a + _np.conjugate(_np.swapaxes(a, -1, -2)))
        w, v = _np.linalg.eigh(a, UPLO="L" if UPLO is None else UPLO)
        return _wrap(w), _wrap(v)

    def __getattr__(self, name):
        return _wrapfn(getattr(_np.linalg, name))


class _FFT:
    def __getattr__(self, name):
        return _wrapfn(getattr(_np.fft, name))


linalg = _Linalg()
fft = _FFT()

pi = _np.pi
newaxis = None
float64 = _np.float64
float32 = _np.float32
complex128 = _np.complex128
complex64 = _np.complex64
int32 = _np.int32
int64 = _np.int64
bool_ = _np.bool_
ndarray = JArray
finfo = _np.finfo
inf = _np.inf


def __getattr__(name):
    obj = getattr(_np, name)
    if callable(obj) and not isinstance(obj, type):
        return _wrapfn(obj)
    return obj
