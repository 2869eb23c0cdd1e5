"""Problem plugins on the CPU: building against the plugin SDK with the
content-addressed cache, the registration checks of the loader, the parameter
checks and the construction checks.  Nothing here launches a kernel: the
plugin's constructor is host code.  Builds go to tests/.native_cache."""
import json
import os
from pathlib import Path

import pytest

from cuda_moea import native
from cuda_moea._lib import MoeaError

HERE = Path(__file__).resolve().parent
PLUGINS = HERE / "native"
CACHE = HERE / ".native_cache"


@pytest.fixture(scope="module")
def spheres_lib():
    return native.build_problem(PLUGINS / "weighted_spheres", cache_dir=CACHE)


def _problem(lib, **params):
    return native.NativeProblem(library=lib, name="WeightedSpheres", dimension=6, objectives=2,
                                lower_bounds=-1.0, upper_bounds=2.0, parameters=params)


def test_build_is_cached_and_the_schema_is_registered(spheres_lib, capsys):
    again = native.build_problem(PLUGINS / "weighted_spheres", cache_dir=CACHE)
    assert again == spheres_lib
    assert native.build_problem(PLUGINS / "weighted_spheres", cache_dir=CACHE, mode="never") == spheres_lib
    s = native.schema(spheres_lib)
    assert s["name"] == "WeightedSpheres"
    assert s["build_id"] == "moea-b200-native-sdk-1"
    p = s["parameters"]
    assert p["shift"] == {"type": "float", "default": 0.5, "description": "center of the second sphere"}
    assert p["weights"]["type"] == "float_list" and p["weights"]["default"] == [1.0, 1.0]
    assert p["constrained"]["type"] == "bool" and p["constrained"]["default"] is False
    assert p["switch_at"]["type"] == "int" and p["switch_at"]["default"] == -1
    assert p["label"]["type"] == "str" and p["label"]["default"] == "WeightedSpheres"
    native.main(["inspect", str(spheres_lib)])
    assert json.loads(capsys.readouterr().out)["name"] == "WeightedSpheres"


def test_parameters_and_construction_are_checked(spheres_lib):
    from cuda_moea.native import NativeInstance
    ok = _problem(spheres_lib, shift=1, weights=[1, 2.5], constrained=True, switch_at=3, label="x")
    inst = NativeInstance(ok._spec())
    assert inst.constraint_count == 1
    del inst
    with pytest.raises(ValueError, match="Unknown native problem parameter"):
        _problem(spheres_lib, nope=1)
    with pytest.raises(ValueError, match="must be float"):
        _problem(spheres_lib, shift="far")
    with pytest.raises(ValueError, match="must be int"):
        _problem(spheres_lib, switch_at=2.5)
    with pytest.raises(ValueError, match="must be bool"):
        _problem(spheres_lib, constrained=1)
    with pytest.raises(ValueError, match="registers 'WeightedSpheres'"):
        native.NativeProblem(library=spheres_lib, name="Other", dimension=6, objectives=2)
    with pytest.raises(ValueError, match="lower bound"):
        native.NativeProblem(library=spheres_lib, name="WeightedSpheres", dimension=2, objectives=2,
                             lower_bounds=1.0, upper_bounds=1.0)
    with pytest.raises(MoeaError, match="asked to fail"):
        NativeInstance(_problem(spheres_lib, throw_at_create=True)._spec())
    with pytest.raises(MoeaError, match="must match the requested dimensions"):
        NativeInstance(_problem(spheres_lib, bad_info=True)._spec())
    with pytest.raises(MoeaError, match="objectives=2"):
        NativeInstance(native.NativeProblem(library=spheres_lib, name="WeightedSpheres", dimension=6,
                                            objectives=3)._spec())


def test_foreign_and_unregistered_libraries_are_refused():
    wrong = native.build_problem(PLUGINS / "wrong_sdk", cache_dir=CACHE)
    with pytest.raises(MoeaError, match="SDK mismatch"):
        native.schema(wrong)
    bare = native.build_problem(PLUGINS / "no_registration", cache_dir=CACHE)
    with pytest.raises(MoeaError, match="Missing cuda_moea_problem_v1"):
        native.schema(bare)
    with pytest.raises(MoeaError, match="Cannot load"):
        native.schema(HERE / "native" / "no_such_library.so")


def test_never_mode_clean_and_export(spheres_lib, tmp_path_factory):
    scratch = CACHE / "scratch_cache"
    native.clear_cache(scratch)
    with pytest.raises(FileNotFoundError):
        native.build_problem(PLUGINS / "no_registration", cache_dir=scratch, mode="never")
    built = native.build_problem(PLUGINS / "no_registration", cache_dir=scratch)
    assert built.is_file()
    native.clear_cache(scratch)
    assert not built.exists()
    out = CACHE / "export_test"
    if out.exists():
        for f in out.iterdir():
            os.remove(f)
    exported = native.export_problem(spheres_lib, out)
    assert native.schema(exported)["name"] == "WeightedSpheres"
    with pytest.raises(FileExistsError):
        native.export_problem(spheres_lib, out)
    with pytest.raises(ValueError):
        native.build_problem(PLUGINS / "weighted_spheres", cache_dir=PLUGINS / "weighted_spheres" / "c")


# The reference's example plugin (examples/native/bi_sphere), compiled unchanged
# against this SDK by oracle/ref/Makefile; present where the reference's sources
# were available to the build.  The cases follow the reference's own plugin
# tests (tests/python/test_native_problem.py:159-232).
BI_SPHERE = HERE.parent / "oracle" / "_ref" / "bi_sphere" / "problem.so"
needs_bi_sphere = pytest.mark.skipif(not BI_SPHERE.is_file(), reason="reference example plugin not built")


def _bi_sphere(**kwargs):
    options = dict(library=BI_SPHERE, name="BiSphere", dimension=7, objectives=2,
                   lower_bounds=-5.0, upper_bounds=5.0)
    options.update(kwargs)
    return native.NativeProblem(**options)


@needs_bi_sphere
def test_reference_plugin_registration_and_algorithm_construction():
    import gc
    import cuda_moea as cm
    p = _bi_sphere(parameters={"offset": 4.0, "constrained": True})
    assert p.schema["name"] == "BiSphere"
    assert p.schema["parameters"]["radius"]["default"] == 3.0
    assert p.schema["parameters"]["offset"]["default"] == 2.0
    assert p.schema["parameters"]["constrained"] == {
        "type": "bool", "default": False, "description": "Enable sum(x*x) <= radius*radius"}
    assert p._spec()["type"] == "NativeProblem"
    for algorithm in (cm.NSGA3, cm.RVEA):
        instance = algorithm(problem=p, population_size=32, max_generations=2, enable_warmup=False)
        assert not instance.initialized
        del instance
    gc.collect()


@needs_bi_sphere
def test_reference_plugin_parameters_do_not_alias():
    first = _bi_sphere(parameters={"offset": 1.0})
    second = _bi_sphere(dimension=129, parameters={"offset": 7.0})
    assert first.library == second.library
    spec = first._spec()
    spec["parameters"]["offset"] = 99
    assert first._spec()["parameters"]["offset"] == 1.0


@needs_bi_sphere
def test_reference_plugin_invalid_parameters_names_and_dimensions():
    import cuda_moea as cm
    for params in ({"offest": 2}, {"offset": True}, {"offset": float("nan")}, {"constrained": 1}):
        with pytest.raises(ValueError):
            _bi_sphere(parameters=params)
    with pytest.raises(ValueError):
        _bi_sphere(name="unknown")
    with pytest.raises(ValueError):
        _bi_sphere(lower_bounds=5.0)
    with pytest.raises(ValueError, match="objectives=2"):
        cm.NSGA3(problem=_bi_sphere(objectives=3))
    # the algorithm checks the specification again
    p = _bi_sphere()
    p._config["parameters"] = {"offset": True}
    with pytest.raises(ValueError, match="Invalid type/value"):
        cm.NSGA3(problem=p)
    p._config["parameters"] = {"radius": -1.0}
    with pytest.raises(ValueError, match="nonnegative"):
        cm.NSGA3(problem=p)
