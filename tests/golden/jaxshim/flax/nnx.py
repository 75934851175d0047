"""``flax.nnx`` stand-in: ``Module`` is a plain object base class."""


class Module:
    def __init__(self, *args, **kwargs):
        pass
