"""Placeholder replaced by the reference-kernel build recipe."""


def build(force: bool = False) -> None:
    raise RuntimeError("reference kernel build not available yet")
