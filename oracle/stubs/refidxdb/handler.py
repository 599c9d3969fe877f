"""Stand-in ``refidxdb.handler.Handler``, TEST ONLY: material I/O is out of scope."""


class Handler:  # noqa: D101
    def __init__(self, *args, **kwargs):
        raise RuntimeError("refidxdb is not available: material database I/O is out of scope")
