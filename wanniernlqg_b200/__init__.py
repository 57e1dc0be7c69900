"""B200-native engine for the WannierNLQG k-mesh response hot path."""
from .model import TightBindingModel, read_wannier_tb, write_wannier_tb  # noqa: F401
from .bundle import (  # noqa: F401
    model_from_operator_bundle,
    read_operator_bundle_components,
    read_operator_bundle_payload,
    read_real_space_operator_bundle,
    read_real_space_operator_bundle_manifest,
    write_model_operator_bundle,
    write_real_space_operator_bundle,
)
