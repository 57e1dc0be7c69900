"""B200-native engine for the WannierNLQG k-mesh response hot path."""
from .model import TightBindingModel, read_wannier_tb, write_wannier_tb  # noqa: F401
