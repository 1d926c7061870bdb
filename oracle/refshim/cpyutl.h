/*
 * Minimal stand-in for the `cpyutl` helper library that the reference extension
 * (j4nr0th/hybridized-solver, `src/*.c`) includes as `<cpyutl.h>`.
 *
 * TEST INFRASTRUCTURE ONLY. The reference pins `cpyutl` as a git submodule
 * (`.gitmodules:1-3`) that is empty in the mounted tree and cannot be fetched
 * offline. Nothing in it does arithmetic: it parses arguments, checks arrays,
 * builds tuples, registers heap types and provides an assert macro. This file
 * restates exactly the API surface the reference calls, written from those call
 * sites (e.g. `src/block_system.c:181-189`, `src/blocks.c:190`,
 * `src/module.c:32-34`), so the reference's own C sources compile unchanged into
 * `oracle/_ref/` and serve as the parity oracle.
 */
#pragma once

#include <Python.h>
#include <numpy/ndarrayobject.h>

#ifdef CPYUTL_ENABLE_ASSERTS
/* A function call rather than an inline fprintf: the reference uses this macro
 * inside OpenMP `default(none)` regions, which reject references to `stderr`. */
void cpyutl_failed_assert(const char *file, int line, const char *fmt, ...);
#define CPYUTL_ASSERT(cond, ...)                                                                                       \
    do                                                                                                                 \
    {                                                                                                                  \
        if (!(cond))                                                                                                   \
            cpyutl_failed_assert(__FILE__, __LINE__, __VA_ARGS__);                                                     \
    } while (0)
#else
#define CPYUTL_ASSERT(cond, ...) ((void)0)
#endif

typedef enum
{
    CPYARG_TYPE_END = 0, /* the zero-initialised `{}` terminator of a spec array */
    CPYARG_TYPE_SSIZE,
    CPYARG_TYPE_PYTHON,
    CPYARG_TYPE_CUSTOM,
} cpyutl_argument_type_t;

typedef struct
{
    cpyutl_argument_type_t type;
    void *p_val;
    const char *kwname;
    int optional;
    PyTypeObject *type_check;
    int (*custom_convert)(PyObject *value, void *p_out, const char *name);
} cpyutl_argument_t;

typedef enum
{
    CPYOUT_TYPE_END = 0,
    CPYOUT_TYPE_PYINT,
    CPYOUT_TYPE_TUPLE,
} cpyutl_output_type_t;

typedef struct
{
    cpyutl_output_type_t type;
    Py_ssize_t value_int;
} cpyutl_output_t;

/* Returns 0 when `arr` has dtype `dtype`, all of `flags`, and (for ndim > 0) the
 * given number of dimensions and extents; otherwise sets ValueError and returns -1. */
int check_input_array(const PyArrayObject *arr, int ndim, const npy_intp *dims, int dtype, int flags, const char *name);

/* Parses a METH_FASTCALL|METH_KEYWORDS argument vector into `spec` (terminated by a
 * zeroed entry). Optional arguments that are absent keep their initial value. */
int parse_arguments_check(cpyutl_argument_t *spec, PyObject *const *args, Py_ssize_t nargs, const PyObject *kwnames);

/* Builds a tuple of Python ints from a zero-terminated output list. */
PyObject *cpyutl_output_create_check(cpyutl_output_type_t type, const cpyutl_output_t *outputs);

/* Creates a heap type bound to `mod` and adds it to the module under its short name. */
PyTypeObject *cpyutl_add_type_from_spec_to_module(PyObject *mod, PyType_Spec *spec, PyObject *bases);
