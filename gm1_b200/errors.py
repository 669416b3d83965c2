"""Typed refusals for unsupported operator branches.

Mirrors the reference's refusal shape (src/cm1core/errors.py:1-20): the
exception names the option, the value given, why running it would produce a
wrong result, and the remedy.
"""

from __future__ import annotations


class CM1Refusal(ValueError):
    def __init__(self, *, code: str, gate: str, option: str, value: object, reason: str, remedy: str):
        self.code = code
        self.gate = gate
        self.option = option
        self.value = value
        self.reason = reason
        self.remedy = remedy
        super().__init__(f"[{code}] {gate}: {option}={value!r} refused: {reason}; remedy: {remedy}")


def refuse(*, code: str, gate: str, option: str, value: object, reason: str, remedy: str) -> None:
    raise CM1Refusal(code=code, gate=gate, option=option, value=value, reason=reason, remedy=remedy)
