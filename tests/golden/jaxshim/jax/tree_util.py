"""``jax.tree_util`` stand-in; golden-vector generation only."""


def register_dataclass(cls=None, **_k):
    if cls is None:
        return lambda c: c
    return cls
