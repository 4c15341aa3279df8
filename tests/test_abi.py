"""C-ABI boundary: the library loads, exports every symbol include/tetfit.h
declares, and reports script errors with the reference's messages."""
import os
import re

import pytest

import tetfit_b200 as tb
from tetfit_b200.cases import FitCase, write_fit_cavity

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "tetfit.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^TF_API\s+[\w\s\*]+?\b(tf_\w+)\(", text, flags=re.M)))


def test_every_declared_symbol_is_exported(product_lib):
    names = declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(product_lib, n), n
    assert set(names) == set(tb._SIGS), "python mirror and header disagree"


def test_open_and_list_simulations(tmp_path, product_lib):
    script = write_fit_cavity(str(tmp_path), FitCase(n=8, steps=5))
    d = tb.Discretization(script)
    assert d.simulations == [1]
    d.close()


@pytest.mark.parametrize("body,line,msg", [
    ("SET type pec\n", 1, "define something before setting variables"),
    ("DEFINE widget 1\n", 1, "can only define one of the following"),
    ("DEFINE bc 1\n  SET type pmx\nEND bc 1\n", 2, "Unrecognized boundary condition type"),
    ("DEFINE source 1\n  SET carrier square\nEND source 1\n", 2, "Unrecognized source carrier"),
    ("DEFINE source 1\n  SET center {1,2,3,4}\nEND source 1\n", 2, "Maximum of three coordinates!"),
    ("DEFINE source 1\n  SET center 1,2,3\nEND source 1\n", 2, "coordinates must be inside braces"),
    ("DEFINE output 1\n  SET mode movie\nEND output 1\n", 2, "Undefined output mode type"),
    ("DEFINE simulation 1\n  SET method leapfrog\nEND simulation 1\n", 2, "Undefined simulation method"),
    ("DEFINE simulation 1\n  SET flavour x\nEND simulation 1\n", 2, "Undefined simulation parameter"),
    ("DEFINE material 1\n  SET epsilon 2\nEND material 2\n", 3, "ending unopened definition"),
    ("DEFINE material 1\n  SET epsilon 2\n", 3, "File ended unexpectedly"),
    ("DEFINE material 1\n  FOO epsilon 2\nEND material 1\n", 2, "Unknown instruction inside define block"),
    ("DEFINE mesh 1\n  SET file does_not_exist.mesh\nEND mesh 1\n", 2, "Mesh input file does not exist"),
])
def test_script_errors_carry_reference_text(tmp_path, product_lib, body, line, msg):
    p = tmp_path / "bad.fdtd"
    p.write_text(body)
    with pytest.raises(tb.TetfitError) as ei:
        tb.Discretization(str(p))
    assert ei.value.code == tb.TF_E_SCRIPT
    assert ei.value.message.startswith(f"Input file error at line {line}: ")
    assert msg in ei.value.message


def test_unknown_label_and_order_errors(tmp_path, product_lib):
    script = write_fit_cavity(str(tmp_path), FitCase(n=8, steps=5))
    d = tb.Discretization(script)
    with pytest.raises(tb.TetfitError) as ei:
        d.step(1)
    assert ei.value.code == tb.TF_E_STATE
    with pytest.raises(tb.TetfitError) as ei:
        d.prepare(7)
    assert ei.value.code == tb.TF_E_ARG
    d.close()


def test_file_digits_out_of_range_is_rejected(tmp_path, product_lib):
    script = write_fit_cavity(str(tmp_path), FitCase(n=8, steps=5))
    d = tb.Discretization(script)
    with pytest.raises(tb.TetfitError) as ei:
        d.prepare(1, file_digits=18)
    assert ei.value.code == tb.TF_E_ARG and "file_digits" in ei.value.message
    d.close()
