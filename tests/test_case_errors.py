"""The loader's error behaviour against the reference's: every malformed document of
tests/golden/case_errors.json (made by make_golden_case_errors.py from the reference's
own loader) raises a ``CaseError`` with the reference's message.  The one difference
allowed: lists of allowed keys or choices also name jaxrans_b200's additions (the domain key
``normal_stretching``, the preconditioner ``line_j_coupled``)."""

from __future__ import annotations

import copy
import json
from pathlib import Path

import pytest

from jaxrans_b200.case import CaseError, apply_override, parse_case

ADDED = ("'normal_stretching', ", "'line_j_coupled', ")
ERRORS = json.loads((Path(__file__).resolve().parent / "golden" / "case_errors.json").read_text())


def without_additions(message: str) -> str:
    for name in ADDED:
        message = message.replace(name, "")
    return message


def mutated(docs, file, path, value):
    docs = copy.deepcopy(docs)
    node = docs[file]
    *head, last = path.split(".")
    for part in head:
        node = node.setdefault(part, {})
    if value == "<delete>":
        node.pop(last, None)
    else:
        node[last] = value
    return docs


def base(label):
    docs = {"case": ERRORS["base_case"], "numerical": ERRORS["base_numerical"]}
    if label == "inviscid":
        docs = mutated(mutated(docs, "case", "freestream.reynolds", "<delete>"), "case", "turbulence", "<delete>")
    return docs


def test_the_base_documents_parse():
    parse_case(*base("viscous").values())
    parse_case(*base("inviscid").values())


@pytest.mark.parametrize("entry", ERRORS["parse"], ids=[e["name"] for e in ERRORS["parse"]])
def test_parse_errors_match_the_reference(entry):
    docs = mutated(base(entry["base"]), entry["file"], entry["path"], entry["value"])
    with pytest.raises(CaseError) as raised:
        parse_case(docs["case"], docs["numerical"])
    assert without_additions(str(raised.value)) == entry["message"]


@pytest.mark.parametrize("entry", ERRORS["override"], ids=[e["assignment"] for e in ERRORS["override"]])
def test_override_errors_match_the_reference(entry):
    with pytest.raises(CaseError) as raised:
        apply_override(copy.deepcopy(base("viscous")), entry["assignment"])
    assert str(raised.value) == entry["message"]
