"""SBML import on CPU (cutauleaping_b200.sbml, replacing SBML2BSW.py): the
converter's tables, the folder it writes read back through the C ABI
(ctl_model_load / ctl_rows_load), the reverse-reaction rule of
SBML2BSW.py get_reactions, and its error paths.  The SBML files under
tests/golden/ were written for these tests."""
import os

import numpy as np
import pytest

import cutauleaping_b200 as ctl
from cutauleaping_b200 import inputs, sbml

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_schlogl_tables_match_the_builtin_model():
    m = sbml.load(os.path.join(GOLDEN, "schlogl_l2.xml"))
    ref = inputs.schlogl(1)
    assert np.array_equal(m.left, ref.left) and np.array_equal(m.right, ref.right)
    assert np.array_equal(m.feed, ref.feed)
    assert np.array_equal(m.x0, ref.X0[0])
    assert np.allclose(m.c, ref.c[0], rtol=0, atol=0)
    assert m.names == ["A_in_cell", "X_in_cell", "B_in_cell"]
    assert np.array_equal(sbml.load(os.path.join(GOLDEN, "schlogl_l2.xml"), reference_feeds=True).feed, [0, 0, 0])


def test_folder_reads_back_through_the_c_abi(tmp_path):
    m = sbml.load(os.path.join(GOLDEN, "schlogl_l2.xml"))
    out = sbml.write_folder(m, str(tmp_path / "f"), sims=5, t_end=2.0, samples=20)
    model = ctl.Model.load(out)
    assert (model.S, model.R, model.ns) == (3, 4, 20)
    X0, c = ctl.load_rows(out, model, 0, 5)
    assert np.array_equal(X0, np.tile(m.x0.astype(np.int32), (5, 1)))
    assert np.array_equal(c, np.tile(m.c.astype(np.float32), (5, 1)))


def test_reversible_reaction_with_global_parameters():
    m = sbml.load(os.path.join(GOLDEN, "dimer_l3.xml"))
    assert m.reactions == ["dimerise", "dimerise (reverse)"]
    assert np.array_equal(m.left, [[2, 0], [0, 1]]) and np.array_equal(m.right, [[0, 1], [2, 0]])
    assert np.array_equal(m.c, [0.002, 0.5])
    assert m.names == ["monomer_in_c", "dimer_in_c"]
    assert np.array_equal(m.x0, [400, 0]) and np.array_equal(m.feed, [0, 0])


@pytest.mark.parametrize("edit,msg", [
    (lambda s: s.replace("</listOfReactions>", "</listOfReactions><listOfRules><assignmentRule variable='kf'/>"
                         "</listOfRules>"), "rules"),
    (lambda s: s.replace('species="D" stoichiometry="1"', 'species="Q" stoichiometry="1"'), "unknown species"),
    (lambda s: s.replace("<ci> kr </ci>", "<ci> kf </ci>"), "rate constant"),  # reversible, one constant
    (lambda s: s.replace("<ci> kf </ci>", "<ci> zz </ci>").replace("<ci> kr </ci>", "<ci> yy </ci>"),
     "no kinetic parameter"),
])
def test_errors(tmp_path, edit, msg):
    src = open(os.path.join(GOLDEN, "dimer_l3.xml")).read()
    p = tmp_path / "bad.xml"
    p.write_text(edit(src))
    with pytest.raises(sbml.SbmlError, match=msg):
        sbml.load(str(p))


def test_command_line(tmp_path, capsys):
    assert sbml.main([os.path.join(GOLDEN, "dimer_l3.xml"), str(tmp_path / "o"), "--sims", "3"]) == 0
    assert open(tmp_path / "o" / "MX_0").read() == "400\t0\n" * 3
    assert sbml.main([str(tmp_path / "missing.xml"), str(tmp_path / "o2")]) == 2


def test_mutated_sbml_raises_only_sbml_errors(tmp_path):
    """Seeded random damage to the two fixtures -- cut, inserted and
    truncated text, odd attribute values (negative, huge, non-numeric,
    infinite), unknown XML encodings -- either imports or raises SbmlError."""
    import random
    srcs = [open(os.path.join(GOLDEN, n)).read() for n in ("schlogl_l2.xml", "dimer_l3.xml")]
    tokens = ["<", ">", "/", "\"", "=", " ", "x", "-1", "1e400", "nan", "2.5", "true", "</model>",
              "<species id=\"q\"/>", "reversible=\"true\"", "stoichiometry=\"-3\"", "stoichiometry=\"1.5\"",
              "<ci> k </ci>", "&amp;", "&bad;"]
    rng = random.Random(5)
    path = str(tmp_path / "m.xml")
    for _ in range(800):
        d = rng.choice(srcs)
        for _ in range(rng.randint(1, 5)):
            i, op = rng.randrange(len(d) + 1), rng.randrange(4)
            if op == 0:
                d = d[:i] + d[i + rng.randint(1, 40):]
            elif op == 1:
                d = d[:i] + rng.choice(tokens) + d[i:]
            elif op == 2:
                a = d.find('"', i)
                b = d.find('"', a + 1)
                if a >= 0 and b > a:
                    d = d[:a + 1] + rng.choice(["", "0", "-5", "abc", "1e308", "inf", "3", "UTFx-8"]) + d[b:]
            else:
                d = d[:i]
        with open(path, "w") as f:
            f.write(d)
        try:
            m = sbml.load(path)
            sbml.write_folder(m, str(tmp_path / "out"), sims=2, t_end=1.0, samples=3)
        except sbml.SbmlError:
            pass
