"""The command-line smoke run (python -m rustatevec_b200): the GHZ output of qsv's CLI
(crates/qsv-cli/src/main.rs:1-31), from the B200 engine."""
import pytest

from rustatevec_b200.__main__ import main

pytestmark = pytest.mark.gpu


def test_ghz_output(built, capsys):
    assert main(["5"]) == 0
    out = capsys.readouterr().out.splitlines()
    assert out[0] == "GHZ(5) — non-negligible outcome probabilities:"
    assert out[1:3] == ["  |00000⟩ : 0.500000", "  |11111⟩ : 0.500000"]
    assert out[3] == "⟨ψ|ψ⟩ = 1.000000" and len(out) == 4


def test_default_width(built, capsys):
    assert main(["not-a-number"]) == 0
    out = capsys.readouterr().out.splitlines()
    assert out[0].startswith("GHZ(4)") and out[1] == "  |0000⟩ : 0.500000"
