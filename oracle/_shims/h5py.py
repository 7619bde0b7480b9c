"""Stand-in for ``h5py`` so the Renormalizer reference imports in this
container when golden fixtures are made.  Test infrastructure only: the
reference touches h5py solely for out-of-core Davidson storage, which the
fixture cases never enable (everything stays in core)."""


class File:  # pragma: no cover - never instantiated by the fixture cases
    def __init__(self, *args, **kwargs):
        raise RuntimeError("h5py stand-in: out-of-core storage is not available")
