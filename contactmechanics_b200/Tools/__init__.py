from .Logger import Logger, quiet, screen  # noqa: F401
