"""Content per arithmetic profile for the GPU tests.

The shader profile (SPEC) reconstructs only frames coded with the regular
8-tap filter — the shaders hold that table alone — and returns
CVP9_ERR_UNSUPPORTED for the others, so its test streams are generated with
interp_filter = EIGHTTAP. The CPU profile (REFCPU) never reads the field.
"""
from oracle.oracle_py import SPEC


def overrides_for(profile, overrides):
    if profile == SPEC and "interp_filter" not in overrides:
        return dict(overrides, interp_filter=0)
    return dict(overrides)


def mix_for(profile, mix):
    return [(p, w, h, overrides_for(profile, ov)) for (p, w, h, ov) in mix]
