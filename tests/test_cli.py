"""The command line's argument handling (no GPU work): the reference's option
names and defaults (CUDA-based/main_CAGR.py:14-23), and the errors for the CPU
mode this library does not have and for unsupported input files."""
import pytest

from cagr_b200.__main__ import main


def test_cpu_mode_is_rejected():
    with pytest.raises(SystemExit, match="no CPU path"):
        main(["orient", "cloud.xyz", "--width_config", "l0", "--cpu"])


def test_input_extension_is_checked():
    with pytest.raises(SystemExit, match="xyz/npy"):
        main(["orient", "cloud.txt", "--width_config", "l0"])


def test_width_config_choices_and_required():
    with pytest.raises(SystemExit):
        main(["orient", "cloud.xyz"])
    with pytest.raises(SystemExit):
        main(["orient", "cloud.xyz", "--width_config", "l9"])
