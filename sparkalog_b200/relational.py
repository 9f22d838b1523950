"""Backend-neutral plan vocabulary of the binary recursive pipeline.

Mirrors crates/sparkalog-relational/src/lib.rs:10-89 (same names and field
meaning), so plans read the same as in the reference.
"""

from __future__ import annotations

import enum
from dataclasses import dataclass, field


class RelationVersion(enum.Enum):
    """relational/src/lib.rs:10-14."""

    FULL = 0
    DELTA = 1
    NEWT = 2


@dataclass(frozen=True, order=True)
class RelationId:
    """relational/src/lib.rs:16-17."""

    value: int


class JoinInput(enum.IntEnum):
    """relational/src/lib.rs:33-37 (the C ABI encodes Left as 0, Right as 1)."""

    LEFT = 0
    RIGHT = 1


@dataclass(frozen=True)
class JoinProjection:
    """relational/src/lib.rs:39-43."""

    input: JoinInput
    column: int


@dataclass(frozen=True)
class BinaryEqualityJoin:
    """A single-key equality join with a binary projected output (relational/src/lib.rs:45-50)."""

    left_key: int
    right_key: int
    output: tuple[JoinProjection, JoinProjection]


@dataclass(frozen=True)
class BinaryDistinct:
    """Sort and deduplicate a projected pair of u32 columns (relational/src/lib.rs:52-56)."""

    columns: tuple[int, int] = (0, 1)


@dataclass(frozen=True)
class SortedBinaryAntiJoin:
    """Set difference of lexicographically sorted binary relations (relational/src/lib.rs:58-63)."""

    left: tuple[int, int] = (0, 1)
    right: tuple[int, int] = (0, 1)


@dataclass(frozen=True)
class SortedBinaryUnion:
    """Set union of lexicographically sorted binary relations (relational/src/lib.rs:65-70)."""

    left: tuple[int, int] = (0, 1)
    right: tuple[int, int] = (0, 1)


class U32Predicate(enum.IntEnum):
    """Comparison of a u32 value with an operand (crates/sparkalog-relational/src/lib.rs:144-164);
    the integer values are the operation codes of the filter ABI."""

    EQ = 0
    NE = 1
    LT = 2
    LE = 3
    GT = 4
    GE = 5

    def matches(self, value: int, operand: int) -> bool:
        return {0: value == operand, 1: value != operand, 2: value < operand, 3: value <= operand,
                4: value > operand, 5: value >= operand}[int(self)]


@dataclass(frozen=True)
class Filter:
    """A filter producing compact row ids (lib.rs:166-171): column, predicate and operand."""

    column: int
    predicate: U32Predicate
    operand: int


@dataclass
class RecursiveRulePlan:
    """One semi-naive binary rule lowered to operators (relational/src/lib.rs:72-82)."""

    target: RelationId
    delta_input: RelationId
    right_input: RelationId
    join: BinaryEqualityJoin
    distinct: BinaryDistinct = BinaryDistinct()
    anti_join: SortedBinaryAntiJoin = SortedBinaryAntiJoin()
    union: SortedBinaryUnion = SortedBinaryUnion()


@dataclass
class RecursiveSccPlan:
    """A strongly connected set of recursive relations (relational/src/lib.rs:84-89)."""

    relations: list[RelationId]
    rules: list[RecursiveRulePlan] = field(default_factory=list)


def path_join() -> BinaryEqualityJoin:
    """path(x, z) :- path(x, y), edge(y, z): DELTA column 1 = edge column 0, output (L.0, R.1)."""
    return BinaryEqualityJoin(
        left_key=1,
        right_key=0,
        output=(JoinProjection(JoinInput.LEFT, 0), JoinProjection(JoinInput.RIGHT, 1)),
    )
