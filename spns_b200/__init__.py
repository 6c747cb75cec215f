"""spns_b200: B200-native pseudospectral time step of SpNS behind the reference's HIT interface."""
from .params import read_params, derive_hit_args, read_initial_field, read_forced_ek, HitArgs, ParamsError  # noqa: F401
