"""Stand-in for ``pyperf``, TEST ONLY (imported by yasfpy/yasf.py:32, unused on the path)."""


class Runner:  # noqa: D101
    def __init__(self, *args, **kwargs):
        pass

    def bench_func(self, *args, **kwargs):  # noqa: D102
        raise RuntimeError("pyperf stand-in: benchmarking through pyperf is not available")
