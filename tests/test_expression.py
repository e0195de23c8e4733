"""The scalar-expression compiler (nxg_expression_compile) against the
reference compiler: identical SSA programs (every instruction, operand,
input, ramp point, seed and rand() site seed, floats bitwise) and identical
error texts, plus the Classic noise($Prefg*k) rewrite against the
reference's Classic plan compiler.  Host only; no GPU."""
import numpy as np
import pytest

from nanoxgen_b200.classic import Expression, ExpressionError

# Every op, both statement forms, comments, line joining, locals, methods,
# ramps of every interpolation, literals of every form.
PROGRAMS = [
    "0.5*(1+0.4*$__nxg_pref_noise_0)*clamp(1-$v,0.2,1)",
    "0.01*(1+0.3*$__nxg_pref_noise_0)",
    "rand()", "rand(3)+rand(1,2)+rand(1,2,3)", "hash($id, 2.5)", "hash(1)*hash(2, 3, 4)",
    "$a = 1; $b = $a*2\n$b + 3 # comment\n", "x = 3; x*x", "$a = 1; a = $a + 1; $a",
    "fit($u, 0, 1, -2, 2)", "rampUI(0,0,1:0.5,1,2:1,0.25,3)", "rampUI(0,-1,0:1,2,1)",
    "rampUI(0.25, 0.5, 3 : 0.5, 0.1, 3 : 0.75, 0.9, 3)",
    "$v > 0.5 ? 1 : ($u < 0.2 ? 2 : 3)", "$u ? $v ? 1 : 2 : 3", "!$u || $v && true", "false == !true",
    "$u->clamp(0, 1)->gamma(2.2)", "$u->min(1)->max(0)", "smoothstep($u,0,1)", "-$u + +$v - -1",
    "contrast($u, 0.3)", "min($u,$v)==max($u,$v)", "1e3 + .5 + 0x10", "$a=2;\n(\n$a\n+\n1)",
    "1 <= 2 >= 0 != 1 < 3 > 2", "$u / $v * $id - $cLength", "2 *\n 3\n - 1", "1\n2", "#only a comment\n5",
    "3 \\n 4", "a = 1\nb = 2\na + b",
    # the source rewriting: CR/LF, blank lines, tabs, comments next to operators,
    # escapes inside literals and strings, a comment at the very end
    "1 +\r\n2", "1\r\n\r\n+ 2", "1\t\n\t* 3", "(\n1\n)\n", "1 # a\n# b\n+ 2",
    "$a = 1 #\n$a", "1\f+\v2", "1.e2 + 2.5E-1 + 0x1p3", "2\\n\\n* 3", "4 # tail",
    "-\n1", "!\n0", "$u\n->clamp(0,1)", "min(\n1,\n2\n)", "1 ?\n2 :\n3", "x = 2 ; ; x",
]

ERRORS = [
    "", "1 +", "foo(1)", "map('x')", "$", "1 & 2", "1 | 2", "'str'", "\"unterminated", "rampUI(0,0,4)",
    "rampUI(0,0,1.5)", "clamp(1,2)", "min(1)", "fit(1,2,3,4)", "(1", "1 2", "1e999", "a", "rand(1,2,3,4)",
    "hash()", "@", "rampUI(0.5,0,1:0.2,0,1)", "$u->(1)", "$u->clamp 1", "$u->clamp(0,1", "rampUI(2,0,1)",
    "rampUI(x)", "rampUI(0 0 1)", "rampUI(0,0,1", "1 ? 2", "$1", "noise($Prefg*6)", "max(1,2,3)",
    # offsets counted in the rewritten text (after comments, escapes, joined lines)
    "1 # c\n @", "a\\n@", "'x#y'", "\"a\\\"b\"", "1 +\n\n @", "2 \\n\\n \\n ~", "(1\n", "1\r\n2 3",
    "'a\\nb'", "caf\xe9", "rampUI(0,0,1 : 1,1)", "rampUI(-0.5,0,1)", "$u->", "1 ==", "x = ", "hash(1,)",
    "2 *# c\n3", "1e\\n5",
]

CLASSIC = [
    "0.5*(1+0.4*noise($Prefg*6))", "noise( $Prefg * -2.5 )*$cLength", "$f = 3;\nnoise($Prefg*$f)",
    "0.3 # noise($Prefg*9)\n+noise($Prefg*6)", "noise($Prefg*6)+noise($Prefg*6.0)+noise($Prefg*7)",
    "0.01*(1+0.3*noise($Prefg*20))", "noise($Prefg*1e1)\\n+1", "$id*0.001+noise($Prefg*+4)",
    "noise ($Prefg*2) + noise($Prefg*2 )", "$f = 2; $f = 5; noise($Prefg * $f)",
]


@pytest.mark.parametrize("source", PROGRAMS)
def test_program_matches_reference(nxg_lib, reference, source):
    theirs, message = reference.compile_expression(source, "length", "SplinePrimitive")
    assert theirs is not None, message
    mine = Expression(source, "length", "SplinePrimitive")
    assert mine.describe() == theirs.describe()


@pytest.mark.parametrize("seed_name", [("", ""), ("width", "SplinePrimitive"), ("mask", "NoiseFXModule")])
def test_rand_site_seeds_follow_the_expression_name(nxg_lib, reference, seed_name):
    name, kind = seed_name
    theirs, _ = reference.compile_expression("rand() + rand(1, 2)", name, kind)
    assert Expression("rand() + rand(1, 2)", name, kind).describe() == theirs.describe()


@pytest.mark.parametrize("source", ERRORS)
def test_error_text_matches_reference(nxg_lib, reference, source):
    theirs, message = reference.compile_expression(source, "length", "SplinePrimitive")
    assert theirs is None
    with pytest.raises(ExpressionError) as err:
        Expression(source, "length", "SplinePrimitive")
    assert str(err.value) == message


@pytest.mark.parametrize("source", CLASSIC)
def test_classic_rewrite_matches_reference_plan(nxg_lib, reference, source):
    plan = reference.classic_plan(length=source)
    assert plan.fallback_reasons == []
    mine = Expression.classic(source, "length")
    assert mine.describe() == plan.program("length").describe()
    np.testing.assert_array_equal(mine.pref_noise_frequencies, plan.info()["pref_noise"])


def test_classic_unsupported_forms_are_refused(nxg_lib, reference):
    # map() needs a PTEX binding this runtime does not have; noise() of any
    # other argument is left for the scalar compiler, which rejects it.
    with pytest.raises(ExpressionError, match="PTEX"):
        Expression.classic("map('a.ptx') * 2", "length")
    plan = reference.classic_plan(length="noise($P*6)")
    with pytest.raises(ExpressionError) as err:
        Expression.classic("noise($P*6)", "length")
    assert plan.fallback_reasons == ["SplinePrimitive.length: " + str(err.value)]


def test_string_seed_matches_reference(nxg_lib, reference):
    from nanoxgen_b200._abi import lib
    reference._expression_prototypes()
    for text in ["", "a", "pSphere1", "lengthSplinePrimitive", "x" * 300]:
        assert lib().nxg_xgen_string_seed(text.encode()) == reference.lib.ref_string_seed(text.encode())


def test_expression_info_and_inputs(nxg_lib):
    e = Expression.classic("0.5*(1+0.4*noise($Prefg*6))*clamp(1-$v,0.2,1)", "length")
    info = e.info()
    assert e.inputs == ["__nxg_pref_noise_0", "v"]
    assert info.pref_noise_count == 1 and info.pref_noise_frequencies[0] == 6.0
    assert info.instruction_count == 14 and info.result == 13


def _random_source(rng) -> str:
    """A random expression over the whole grammar, with random blanks, line
    breaks, comments and escapes between tokens (some inputs are invalid on
    purpose)."""
    atoms = ["1", "2.5", ".5", "3e2", "0x10", "$u", "$v", "$id", "$a", "a", "true", "false", "'s'",
             "rand()", "rand(1, 2)", "hash($id, 3)", "min($u, 0.3)", "fit($v, 0, 1, 2, 3)",
             "rampUI(0, 0, 1 : 1, 1, 2)", "clamp($u, 0, 1)", "$u->gamma(2)"]
    binary = ["+", "-", "*", "/", "<", "<=", ">", ">=", "==", "!=", "&&", "||"]
    gaps = [" ", "", "  ", "\t", "\n", "\\n", " # note\n", "\r\n", "\n\n"]

    def value(depth):
        r = rng.random()
        if depth > 3 or r < 0.3:
            return str(rng.choice(atoms))
        if r < 0.6:
            return value(depth + 1) + rng.choice(gaps) + str(rng.choice(binary)) + rng.choice(gaps) + value(depth + 1)
        if r < 0.7:
            return str(rng.choice(["-", "!", "+"])) + value(depth + 1)
        if r < 0.8:
            return "(" + rng.choice(gaps) + value(depth + 1) + rng.choice(gaps) + ")"
        return value(depth + 1) + " ?" + rng.choice(gaps) + value(depth + 1) + " :" + rng.choice(gaps) + value(depth + 1)

    statements = []
    if rng.random() < 0.5:
        statements.append("$a = " + value(1))
    statements.append(value(0))
    return str(rng.choice([";", "\n", "; "])).join(statements)


def test_random_sources_match_reference(nxg_lib, reference):
    """400 seeded random sources: the same program or the same error text."""
    rng = np.random.default_rng(20261204)
    compiled = 0
    for _ in range(400):
        source = _random_source(rng)
        theirs, message = reference.compile_expression(source, "width", "SplinePrimitive")
        if theirs is None:
            with pytest.raises(ExpressionError) as err:
                Expression(source, "width", "SplinePrimitive")
            assert str(err.value) == message, source
        else:
            assert Expression(source, "width", "SplinePrimitive").describe() == theirs.describe(), source
            compiled += 1
    assert 100 < compiled < 400, compiled
