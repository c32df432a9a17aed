"""GPU entry point of the command line (``main_gpu``)."""

from .main import main_gpu

__all__ = ["main_gpu"]
