"""ekpnp -- B200 EK-PNP channel solver (Python host side over libekpnp.so)."""
from ._lib import (EkError, EkParams, FLAG_EXPLICIT_E, FLAG_FORCE, FLAG_MOMENTS_EVERY_STEP,
                   FLAG_REST_QUIRK, STORE_F16, STORE_F32, STORE_F64, lib)
from .batch import Batch
from .channel import FIELD_NAMES, Channel, device_count, set_device
from .params import (BATCH_NX, WORKLOADS, batch_noisy_states, batch_specs, channel_params,
                     helmholtz_smoluchowski, noisy_uniform_state, spec_params, workload_params)

__all__ = ["BATCH_NX", "Batch", "Channel", "EkError", "EkParams", "FIELD_NAMES", "STORE_F16", "STORE_F32",
           "STORE_F64", "FLAG_EXPLICIT_E", "FLAG_FORCE", "FLAG_MOMENTS_EVERY_STEP", "FLAG_REST_QUIRK",
           "WORKLOADS", "batch_noisy_states", "batch_specs", "channel_params", "device_count", "helmholtz_smoluchowski", "lib",
           "noisy_uniform_state", "set_device", "spec_params", "workload_params"]
