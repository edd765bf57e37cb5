"""``jax.lax`` stand-in (eager ``cond``); golden-vector generation only."""
_NO = object()


def cond(pred, true_fun, false_fun, *operands, operand=_NO):
    if operand is not _NO:
        operands = (operand,)
    return true_fun(*operands) if bool(pred) else false_fun(*operands)
