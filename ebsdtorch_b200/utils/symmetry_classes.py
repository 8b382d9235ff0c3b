"""Space group / point group -> Laue group id (1-11), the mapping of
ebsdtorch/utils/symmetry_classes.py:4-64.

The space-group thresholds are the reference's, kept for drop-in parity. They
follow the International Tables except at 194 (P6_3/mmc), which the
reference's ``space_group > 193`` test assigns to class 10 (cubic low) rather
than 9 (hexagonal high); pass ``laue_group=9`` explicitly for that group."""

from __future__ import annotations

import bisect

# first space group number of Laue classes 1..11, as the reference's thresholds
_FIRST_SPACE_GROUP = [1, 3, 16, 75, 89, 143, 156, 168, 177, 194, 207]

_POINT_GROUPS = {
    11: ("m3-m", "4-3m", "432"),
    10: ("m3-", "23"),
    9: ("6/mmm", "6-m2", "6mm", "622"),
    8: ("6/m", "6-", "6"),
    7: ("3-m", "3m", "32"),
    6: ("3-", "3"),
    5: ("4/mmm", "4-2m", "4mm", "422"),
    4: ("4/m", "4-", "4"),
    3: ("mmm", "mm2", "222"),
    2: ("2/m", "m", "2"),
    1: ("1-", "1"),
}
_PG_TO_LAUE = {pg: laue for laue, pgs in _POINT_GROUPS.items() for pg in pgs}


def space_group_to_laue(space_group: int) -> int:
    if space_group < 1 or space_group > 230:
        raise ValueError("The space group must be between 1 and 230 inclusive.")
    return bisect.bisect_right(_FIRST_SPACE_GROUP, int(space_group))


def point_group_to_laue(point_group: str) -> int:
    if point_group not in _PG_TO_LAUE:
        raise ValueError(
            "The point group symbol is not recognized, as one of, "
            + ", ".join(pg for laue in range(11, 0, -1) for pg in _POINT_GROUPS[laue])
        )
    return _PG_TO_LAUE[point_group]
