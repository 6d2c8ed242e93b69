"""CPU checks of the C ABI library: it loads, exports every function include/gp5cu.h
declares, and reports errors as status codes (no device work is attempted here)."""
import ctypes
import os

from gp5_b200 import _abi


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(_abi.LIB_PATH)
    names = _abi.header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_status_strings_and_defaults():
    L = _abi.lib()
    assert L.gp5cu_version() >= 10000
    assert L.gp5cu_status_string(0) == b"ok"
    assert L.gp5cu_status_string(3).startswith(b"non-finite")
    d = _abi.FunctionalDesc()
    L.gp5cu_functional_desc_init(ctypes.byref(d))
    # reference defaults: LHY constants -3 and 5/2 (functional.cpp:118), unit masses
    assert d.kind == _abi.GP5_FUNC_LHY and d.c3 == -3.0 and d.c4 == 2.5
    assert list(d.masses) == [1.0, 1.0] and d.potential == _abi.GP5_POT_NONE


def test_argument_errors_without_device():
    L = _abi.lib()
    # NULL out pointer and bad arguments are rejected before any CUDA call
    rc = L.gp5cu_plan_create(None, (ctypes.c_int * 3)(8, 8, 8), (ctypes.c_double * 3)(-1, -1, -1),
                             (ctypes.c_double * 3)(1, 1, 1), 1, 0, 0)
    assert rc == _abi.GP5_ERR_ARG
    h = ctypes.c_void_p()
    rc = L.gp5cu_plan_create(ctypes.byref(h), (ctypes.c_int * 3)(8, 8, 8), (ctypes.c_double * 3)(-1, -1, -1),
                             (ctypes.c_double * 3)(1, 1, 1), 3, 0, 0)
    assert rc == _abi.GP5_ERR_ARG and b"ncomp" in L.gp5cu_last_error()
    rc = L.gp5cu_plan_create(ctypes.byref(h), (ctypes.c_int * 3)(8, 1, 8), (ctypes.c_double * 3)(-1, -1, -1),
                             (ctypes.c_double * 3)(1, 1, 1), 1, 0, 0)
    assert rc == _abi.GP5_ERR_ARG
    rc = L.gp5cu_stepper_advance(None, None, 1)
    assert rc == _abi.GP5_ERR_ARG


def test_every_declared_function_has_a_ctypes_prototype():
    L = _abi.lib()
    names = _abi.header_functions()
    unbound = [n for n in names if getattr(L, n).argtypes is None]
    assert not unbound, unbound


def test_new_entry_points_reject_bad_arguments_without_device():
    L = _abi.lib()
    k = ctypes.c_int()
    assert L.gp5cu_decompose(None, None, 0, 0.5, None, ctypes.byref(k)) == _abi.GP5_ERR_ARG
    assert L.gp5cu_decompose_host(None, None, 0, 0.5, None, ctypes.byref(k)) == _abi.GP5_ERR_ARG
    assert L.gp5cu_plan_get_tiles(None, None) == _abi.GP5_ERR_ARG
    assert L.gp5cu_stepper_set_compensation(None, 1) == _abi.GP5_ERR_ARG
    assert L.gp5cu_mlp_forward(None, None, 1, None) == _abi.GP5_ERR_ARG
    assert L.gp5cu_gemm_bf16(None, 1, 1, None, 1, 1, None, 1, 1, 1, 1, None) == _abi.GP5_ERR_ARG
    assert L.gp5cu_batch_set_method(None, _abi.GP5_BATCH_PRECOND, 0.5) == _abi.GP5_ERR_ARG
    assert L.gp5cu_init_gaussian(None, None, 0, None) == _abi.GP5_ERR_ARG


def test_reference_facing_bindings_expose_the_extensions():
    import inspect

    from gp5_b200 import gp, gpCpp
    assert hasattr(gpCpp.timeStepper, "setCompensation") and hasattr(gpCpp, "decomposition")
    assert "compensate" in inspect.signature(gp.stepper.__init__).parameters
    assert hasattr(gp.stepper, "setCompensation")


def test_header_is_plain_c_and_links(tmp_path):
    """include/gp5cu.h compiles as C99 and a C caller links against libgp5cu.so (no run: the
    program would need a GPU)."""
    import shutil
    import subprocess

    gcc = shutil.which("gcc")
    if gcc is None:
        import pytest
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "caller.c"
    src.write_text(r'''
#include <stdio.h>
#include "gp5cu.h"
int main(void) {
    gp5cu_plan *plan = NULL;
    const int shape[3] = {64, 64, 64};
    const double left[3] = {-10, -10, -10}, right[3] = {10, 10, 10};
    if (gp5cu_plan_create(&plan, shape, left, right, 1, GP5_C128, 0) != GP5_OK) {
        fprintf(stderr, "%s\n", gp5cu_last_error());
        return 1;
    }
    gp5cu_functional_desc d;
    gp5cu_functional_desc_init(&d);
    d.kind = GP5_FUNC_GP; d.has_couplings = 1; d.couplings[0] = 1.0;
    d.potential = GP5_POT_HARMONIC; d.omegas[0][0] = d.omegas[0][1] = d.omegas[0][2] = 1.0;
    gp5cu_functional *f = NULL;
    gp5cu_stepper *st = NULL;
    void *psi = NULL;
    gp5cu_functional_create(plan, &d, &f);
    gp5cu_stepper_create(f, GP5_STEP_RK4, 1e-3, 1, &st);
    gp5cu_field_alloc(plan, &psi);
    gp5cu_stepper_advance(st, psi, 10);
    gp5cu_observables_t ob;
    gp5cu_observables(f, psi, &ob);
    printf("E = %g\n", ob.energy);
    gp5cu_field_free(plan, psi);
    gp5cu_stepper_destroy(st);
    gp5cu_functional_destroy(f);
    return gp5cu_plan_destroy(plan);
}
''')
    lib = os.path.join(root, "gp5_b200")
    r = subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", "-I", os.path.join(root, "include"), str(src),
                        "-L", lib, "-lgp5cu", "-Wl,-rpath," + lib, "-o", str(tmp_path / "caller")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
