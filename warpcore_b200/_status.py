"""warpcore::Status (status.cuh:16-214) as a Python value type.

The bit values are the reference's ABI.  ``~`` keeps the reference's
definition ``(~s) ^ 0xFFF`` (status.cuh:142-146), which the ReturnBoolean
status handler relies on.
"""

_NAMES = [
    "unknown_error", "probing_length_exceeded", "invalid_configuration",
    "invalid_key", "duplicate_key", "key_not_found", "index_overflow",
    "out_of_memory", "not_initialized", "dry_run", "invalid_phase_overlap",
    "max_values_for_key_reached", "invalid_value",
]
_MASK = 0xFFF


class Status:
    __slots__ = ("_s",)

    def __init__(self, s=0):
        self._s = int(s) & 0xFFFFFFFF

    def base(self):
        return self._s

    def __int__(self):
        return self._s

    @staticmethod
    def none():
        return Status(0)

    @staticmethod
    def all():
        return Status(_MASK)

    @staticmethod
    def error_mask():
        return Status((1 << 0) | (1 << 2) | (1 << 6) | (1 << 7) | (1 << 8) | (1 << 10))

    @staticmethod
    def warning_mask():
        return Status.all() - Status.error_mask()

    def get_errors(self):
        return Status(self._s & Status.error_mask()._s)

    def get_warnings(self):
        return Status(self._s & Status.warning_mask()._s)

    def has_any(self, s=None):
        m = _MASK if s is None else int(s)
        return (self._s & m) != 0

    def has_all(self, s=None):
        m = _MASK if s is None else int(s)
        return (self._s & m) == m

    def has_any_errors(self):
        return self.has_any(Status.error_mask())

    def has_any_warnings(self):
        return self.has_any(Status.warning_mask())

    def __invert__(self):
        return Status(((~self._s) & 0xFFFFFFFF) ^ _MASK)

    def __add__(self, o):
        return Status(self._s | int(o))

    def __sub__(self, o):
        return Status(self._s - (self._s & int(o)))

    def __eq__(self, o):
        return self._s == int(o)

    def __hash__(self):
        return hash(self._s)

    def __bool__(self):
        return self._s != 0

    def names(self):
        return [n for i, n in enumerate(_NAMES) if self._s & (1 << i)]

    def __repr__(self):
        return "Status(%s)" % (", ".join(self.names()) or "none")


def _make_factory(bit):
    return staticmethod(lambda: Status(1 << bit))


def _make_has(bit):
    return lambda self: bool(self._s & (1 << bit))


for _i, _n in enumerate(_NAMES):
    setattr(Status, _n, _make_factory(_i))
    setattr(Status, "has_" + _n, _make_has(_i))
