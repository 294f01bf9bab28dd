"""Exceptions named after the reference's Julia ones."""


class ArgumentError(ValueError):
    """Julia's ArgumentError: an invalid argument value."""


class DimensionMismatch(ValueError):
    """Julia's DimensionMismatch: array shapes that do not fit the grid or each other."""
