"""Test double for matplotlib, which this image does not ship: the
reference's experiment drivers (scripts/common.py) import it at module level
and plot their histories.  Plotting is no part of what the driver tests
check, so every call here records nothing and draws nothing."""


def use(backend, *args, **kwargs):
    return None
