"""Stand-in for the ``opt_einsum`` 3.3 package, used ONLY to import the
Renormalizer reference inside this container when golden fixtures are made.

Test infrastructure: nothing in the product imports this module.

opt_einsum.contract(subscripts, *operands) evaluates an Einstein sum along a
cost-optimal pairwise path; contract_expression(subscripts, *shapes_or_arrays,
constants=[...]) returns a callable that takes the non-constant operands.  Both
are restated on top of numpy.einsum with the optimal path search and its
memory cap lifted (numpy's default cap otherwise forces the naive loop).
"""
import numpy as np

_OPT = ("optimal", 1e13)


def _np_optimize(kwargs):
    kwargs = dict(kwargs)
    kwargs.pop("backend", None)
    opt = kwargs.pop("optimize", None)
    if opt in (None, True, "optimal", "dp", "auto-hq", "auto", "greedy"):
        opt = _OPT
    return opt, kwargs


def contract(*args, **kwargs):
    opt, kwargs = _np_optimize(kwargs)
    return np.einsum(*args, optimize=opt, **kwargs)


def contract_expression(subscripts, *shapes, constants=(), **kwargs):
    opt, kwargs = _np_optimize(kwargs)
    constants = list(constants)
    fixed = {i: shapes[i] for i in constants}
    n = len(shapes)
    cache = {}

    def expr(*arrays, **kw):
        kw.pop("backend", None)
        ops = []
        it = iter(arrays)
        for i in range(n):
            ops.append(fixed[i] if i in fixed else next(it))
        key = tuple(o.shape for o in ops)
        if key not in cache:
            cache[key] = np.einsum_path(subscripts, *ops, optimize=opt)[0]
        return np.einsum(subscripts, *ops, optimize=cache[key])

    return expr


def contract_path(subscripts, *operands, optimize="auto", **kwargs):
    """(path, info) like opt_einsum.contract_path, for callers that only plan
    (torch.einsum consults an importable opt_einsum): numpy's optimal path
    on shape-only placeholders, as a list of operand-index tuples."""
    shapes = [tuple(o.shape) for o in operands]
    ops = [np.lib.stride_tricks.as_strided(np.zeros(1), shape=sh, strides=(0,) * len(sh)) for sh in shapes]
    path, info = np.einsum_path(subscripts, *ops, optimize=_OPT)
    return [tuple(p) for p in path[1:]], info
