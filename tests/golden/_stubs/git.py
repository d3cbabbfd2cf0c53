"""Stand-in for gitpython: the reference generator only asks for a short
commit hash (util/gen_1band_unified_hub.py:17-21), which it stores in
/metadata/commit.  The engine's consistency check compares that string."""


class _Git:
    def rev_parse(self, *args, **kwargs):
        return "refgen0"


class Repo:
    def __init__(self, *args, **kwargs):
        self.git = _Git()
        self.head = None
