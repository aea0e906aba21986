"""The MPMD application's host side without a GPU: input decks (Teuchos ParameterList XML)
and PlatoEngine operation files parse, resolve against the generated mesh and fail with the
reference's messages (src/Analyze_App.cpp, src/EssentialBCs.hpp, src/helmholtz/
HelmholtzResidual.hpp, src/PlatoProblemFactory.hpp) on the mistakes the reference rejects."""
from pathlib import Path

import pytest

from platoanalyze_b200 import capi
from platoanalyze_b200.app import deck_text, validate

DECKS = Path(__file__).resolve().parent / "decks"
CANT = (DECKS / "cantilever.xml").read_text()
OPS = (DECKS / "operations.xml").read_text()
FILT = (DECKS / "filter.xml").read_text()
FOPS = (DECKS / "filter_operations.xml").read_text()


def fails(deck, ops, status, words):
    with pytest.raises(capi.PlatoError) as e:
        validate(deck, ops)
    assert e.value.status == status, str(e.value)
    assert words in str(e.value), str(e.value)


def test_decks_validate_from_text_and_files():
    validate(CANT, OPS)
    validate(FILT, FOPS)
    validate("cantilever.xml", "operations.xml", base_dir=str(DECKS))


def test_deck_text_shows_the_parsed_tree():
    t = deck_text(CANT)
    assert "Input Mesh (string) = box:12,6,6:2.0,1.0,1.0" in t
    assert "\n  Self-Adjoint (bool) = true\n" in t
    assert "\n      Values (Array(double)) = {0.0, -1.0, 0.0}\n" in t
    t = deck_text("<ParameterList name='a'><Parameter name='s' type='string' value='x &lt;&amp;&gt; &#65;'/>"
                  "<!-- comment --><ParameterList name='b'/></ParameterList>")
    assert "s (string) = x <&> A" in t and "b:" in t


@pytest.mark.parametrize("xml,words", [
    ("<ParameterList name='a'><Parameter name='x' type='int' value='1'/>", "unterminated element"),
    ("<ParameterList name='a'>\n<Parameter name='x' type='int' value='1'></ParameterLst>", "XML line 2"),
    ("<ParameterList name='a'><Parameter name='x' type='int' value='1'/><Parameter name='x' type='int' value='2'/>"
     "</ParameterList>", "defined twice"),
    ("<ParameterList name='a'><Parameter name='x' type='int'/></ParameterList>", "needs name, type and value"),
    ("<ParameterList name='a'><Parameter name='x' type='string' value='&bogus;'/></ParameterList>", "unknown entity"),
])
def test_malformed_decks(xml, words):
    with pytest.raises(capi.PlatoError) as e:
        deck_text(xml)
    assert e.value.status == capi.BAD_INPUT and words in str(e.value)


@pytest.mark.parametrize("old,new,status,words", [
    ('<Parameter name="Input Mesh" type="string" value="box:12,6,6:2.0,1.0,1.0"/>', "", capi.BAD_INPUT,
     "'Input Mesh' keyword was not defined"),
    ('value="box:12,6,6:2.0,1.0,1.0"', 'value="part.exo"', capi.BAD_INPUT, "cannot open 'part.exo'"),
    ('value="box:12,6,6:2.0,1.0,1.0"', 'value="box:12,6"', capi.BAD_INPUT, "three cell counts"),
    ('<Parameter name="Sides" type="string" value="x+"/>', '<Parameter name="Sides" type="string" value="q+"/>',
     capi.BAD_INPUT, "no side set 'q+'"),
    ('value="Zero Value"/>\n        <Parameter name="Index" type="int" value="1"/>',
     'value="Mostly Zero"/>\n        <Parameter name="Index" type="int" value="1"/>', capi.BAD_INPUT,
     "Boundary Condition type invalid"),
    ('<Parameter name="Index" type="int" value="2"/>', '<Parameter name="Index" type="int" value="3"/>',
     capi.BAD_INPUT, "Index out of range"),
    ('value="Elliptic"/>', 'value="Hyperbolic"/>', capi.NOT_SUPPORTED,
     "'PDE Constraint' of type 'hyperbolic' is not supported."),
    ('<Parameter name="Physics" type="string" value="Mechanical"/>',
     '<Parameter name="Physics" type="string" value="Thermal"/>', capi.NOT_SUPPORTED, "Physics 'Thermal'"),
    ('<Parameter name="Exponent" type="double" value="3.0"/>\n          <Parameter name="Minimum Value" '
     'type="double" value="1.0e-9"/>\n        </ParameterList>\n      </ParameterList>\n      <ParameterList '
     'name="Material Volume">',
     '<Parameter name="Exponent" type="double" value="2.0"/>\n          <Parameter name="Minimum Value" '
     'type="double" value="1.0e-9"/>\n        </ParameterList>\n      </ParameterList>\n      <ParameterList '
     'name="Material Volume">', capi.NOT_SUPPORTED, "must equal the PDE's"),
    ('<Parameter name="Type" type="string" value="SIMP"/>\n        <Parameter name="Exponent" type="double" '
     'value="3.0"/>\n        <Parameter name="Minimum Value" type="double" value="1.0e-9"/>\n      </ParameterList>\n'
     '    </ParameterList>\n    <ParameterList name="Criteria">',
     '<Parameter name="Type" type="string" value="RAMP"/>\n        <Parameter name="Exponent" type="double" '
     'value="3.0"/>\n        <Parameter name="Minimum Value" type="double" value="1.0e-9"/>\n      </ParameterList>\n'
     '    </ParameterList>\n    <ParameterList name="Criteria">', capi.NOT_SUPPORTED, "only SIMP is built"),
    ('<Parameter name="Youngs Modulus" type="double" value="1.0"/>', "", capi.BAD_INPUT,
     "parameter 'Youngs Modulus' missing"),
    ('value="{0.0, -1.0, 0.0}"', 'value="{0.0, -1.0}"', capi.BAD_INPUT, "'Values' needs 3 entries"),
    ('<Parameter name="Tolerance" type="double" value="1.0e-12"/>',
     '<Parameter name="Tolerance" type="double" value="tight"/>', capi.BAD_INPUT, "not a number"),
])
def test_cantilever_deck_errors(old, new, status, words):
    assert old in CANT
    fails(CANT.replace(old, new, 1), OPS, status, words)


@pytest.mark.parametrize("old,new,words", [
    ("<Criterion>Compliance</Criterion>", "<Criterion>Nope</Criterion>", "no criterion 'Nope'"),
    ("<Criterion>Compliance</Criterion>", "", "Required keyword ('Criterion') missing."),
    ("<ArgumentName>Objective Value</ArgumentName>", "", "'ArgumentName' missing"),
    ("<Name>Compute Objective</Name>", "<Name>Compute Displacement Solution</Name>", "defined twice"),
    ("<ArgumentName>Constraint Gradient</ArgumentName>", "<ArgumentName>Objective Gradient</ArgumentName>",
     "already belongs to criterion"),
    ("<Function>ComputeSolution</Function>\n  <Name>Compute Scaled",
     "<Function>ComputeSolution</Function>\n  <Parameter><ArgumentName>Tip Load Y</ArgumentName></Parameter>\n"
     "  <Name>Compute Scaled", "ArgumentNames must be unique."),
])
def test_operation_errors(old, new, words):
    assert old in OPS
    fails(CANT, OPS.replace(old, new, 1), capi.BAD_INPUT, words)


def test_filter_deck_errors():
    no_params = FILT[:FILT.index('<ParameterList name="Parameters">')] + "</ParameterList>\n</ParameterList>\n"
    fails(no_params, FOPS, capi.BAD_INPUT, "NO PARAMETERS SUBLIST WAS PROVIDED FOR THE HELMHOLTZ FILTER.")
    fails(FILT.replace("{x-}", "{left}"), FOPS, capi.BAD_INPUT, "no side set 'left'")
    fails(FILT.replace('value="0.15"', 'value="-0.15"'), FOPS, capi.BAD_INPUT, "'Length Scale' must be positive")
