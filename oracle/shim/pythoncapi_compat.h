/*
 * Minimal stand-in for the `pythoncapi_compat.h` header that the reference
 * expects from its (unpopulated) `vendored/pythoncapi_compat` git submodule.
 *
 * Test infrastructure only: used when compiling the reference's own
 * `roughpy.compute` CPython extension from its sources into `oracle/_ref/`.
 * The reference sources need exactly one function that is missing from the
 * CPython 3.12 C API: `PyLong_AsInt32` (added to CPython in 3.14).
 *
 * Semantics follow the CPython 3.14 documentation: convert `obj` to a C
 * int32_t, store it in `*value` and return 0; on overflow or a non-integer
 * argument set an exception and return -1.
 */
#ifndef RPYB_ORACLE_PYTHONCAPI_COMPAT_SHIM_H
#define RPYB_ORACLE_PYTHONCAPI_COMPAT_SHIM_H

#include <Python.h>
#include <stdint.h>

#if PY_VERSION_HEX < 0x030E0000
static inline int PyLong_AsInt32(PyObject* obj, int32_t* value)
{
    long v = PyLong_AsLong(obj);
    if (v == -1 && PyErr_Occurred()) {
        return -1;
    }
    if (v < INT32_MIN || v > INT32_MAX) {
        PyErr_SetString(PyExc_OverflowError,
                        "Python int too large to convert to int32_t");
        return -1;
    }
    *value = (int32_t) v;
    return 0;
}
#endif

#endif /* RPYB_ORACLE_PYTHONCAPI_COMPAT_SHIM_H */
