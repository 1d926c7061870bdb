/*
 * Implementation of the `cpyutl` stand-in declared in cpyutl.h.
 * TEST INFRASTRUCTURE ONLY: linked with the reference's sources into the
 * oracle extension under `oracle/_ref/`; never part of the product.
 */
#define PY_ARRAY_UNIQUE_SYMBOL _mod
#define NO_IMPORT_ARRAY
#define NPY_NO_DEPRECATED_API NPY_1_7_API_VERSION
#include "cpyutl.h"

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

void cpyutl_failed_assert(const char *file, int line, const char *fmt, ...)
{
    va_list args;
    va_start(args, fmt);
    fprintf(stderr, "cpyutl assertion failed at %s:%d: ", file, line);
    vfprintf(stderr, fmt, args);
    fputc('\n', stderr);
    va_end(args);
    abort();
}

int check_input_array(const PyArrayObject *arr, int ndim, const npy_intp *dims, int dtype, int flags, const char *name)
{
    if (PyArray_TYPE(arr) != dtype)
    {
        PyErr_Format(PyExc_ValueError, "Array %s has dtype %d, expected %d.", name, PyArray_TYPE(arr), dtype);
        return -1;
    }
    if ((PyArray_FLAGS(arr) & flags) != flags)
    {
        PyErr_Format(PyExc_ValueError, "Array %s does not have the required flags.", name);
        return -1;
    }
    if (ndim == 0)
        return 0;
    if (PyArray_NDIM(arr) != ndim)
    {
        PyErr_Format(PyExc_ValueError, "Array %s has %d dimensions, expected %d.", name, PyArray_NDIM(arr), ndim);
        return -1;
    }
    for (int i = 0; i < ndim; ++i)
    {
        if (PyArray_DIM(arr, i) != dims[i])
        {
            PyErr_Format(PyExc_ValueError, "Array %s has extent %zd in dimension %d, expected %zd.", name,
                         (Py_ssize_t)PyArray_DIM(arr, i), i, (Py_ssize_t)dims[i]);
            return -1;
        }
    }
    return 0;
}

int parse_arguments_check(cpyutl_argument_t *spec, PyObject *const *args, Py_ssize_t nargs, const PyObject *kwnames)
{
    enum
    {
        MAX_ARGS = 32
    };
    Py_ssize_t count = 0;
    while (spec[count].type != CPYARG_TYPE_END)
        ++count;
    if (count > MAX_ARGS)
    {
        PyErr_SetString(PyExc_SystemError, "Too many arguments in the specification.");
        return -1;
    }
    if (nargs > count)
    {
        PyErr_Format(PyExc_TypeError, "Expected at most %zd positional arguments, got %zd.", count, nargs);
        return -1;
    }
    PyObject *given[MAX_ARGS] = {0};
    for (Py_ssize_t i = 0; i < nargs; ++i)
        given[i] = args[i];
    const Py_ssize_t nkw = kwnames ? PyTuple_GET_SIZE((PyObject *)kwnames) : 0;
    for (Py_ssize_t k = 0; k < nkw; ++k)
    {
        const char *kw = PyUnicode_AsUTF8(PyTuple_GET_ITEM((PyObject *)kwnames, k));
        if (!kw)
            return -1;
        Py_ssize_t i = 0;
        while (i < count && strcmp(kw, spec[i].kwname) != 0)
            ++i;
        if (i == count)
        {
            PyErr_Format(PyExc_TypeError, "Unexpected keyword argument '%s'.", kw);
            return -1;
        }
        if (given[i])
        {
            PyErr_Format(PyExc_TypeError, "Argument '%s' given more than once.", kw);
            return -1;
        }
        given[i] = args[nargs + k];
    }
    for (Py_ssize_t i = 0; i < count; ++i)
    {
        PyObject *value = given[i];
        if (!value)
        {
            if (spec[i].optional)
                continue;
            PyErr_Format(PyExc_TypeError, "Missing required argument '%s'.", spec[i].kwname);
            return -1;
        }
        switch (spec[i].type)
        {
        case CPYARG_TYPE_SSIZE: {
            const Py_ssize_t v = PyNumber_AsSsize_t(value, PyExc_OverflowError);
            if (v == -1 && PyErr_Occurred())
                return -1;
            *(Py_ssize_t *)spec[i].p_val = v;
            break;
        }
        case CPYARG_TYPE_PYTHON:
            if (spec[i].optional && value == Py_None)
                continue;
            if (spec[i].type_check && !PyObject_TypeCheck(value, spec[i].type_check))
            {
                PyErr_Format(PyExc_TypeError, "Argument '%s' must be of type %s.", spec[i].kwname,
                             spec[i].type_check->tp_name);
                return -1;
            }
            *(PyObject **)spec[i].p_val = value;
            break;
        case CPYARG_TYPE_CUSTOM:
            if (spec[i].custom_convert(value, spec[i].p_val, spec[i].kwname) < 0)
                return -1;
            break;
        default:
            PyErr_SetString(PyExc_SystemError, "Unknown argument type in the specification.");
            return -1;
        }
    }
    return 0;
}

PyObject *cpyutl_output_create_check(cpyutl_output_type_t type, const cpyutl_output_t *outputs)
{
    (void)type;
    Py_ssize_t count = 0;
    while (outputs[count].type != CPYOUT_TYPE_END)
        ++count;
    PyObject *tuple = PyTuple_New(count);
    if (!tuple)
        return NULL;
    for (Py_ssize_t i = 0; i < count; ++i)
    {
        PyObject *item = PyLong_FromSsize_t(outputs[i].value_int);
        if (!item)
        {
            Py_DECREF(tuple);
            return NULL;
        }
        PyTuple_SET_ITEM(tuple, i, item);
    }
    return tuple;
}

PyTypeObject *cpyutl_add_type_from_spec_to_module(PyObject *mod, PyType_Spec *spec, PyObject *bases)
{
    PyTypeObject *type = (PyTypeObject *)PyType_FromModuleAndSpec(mod, spec, bases);
    if (!type)
        return NULL;
    if (PyModule_AddType(mod, type) < 0)
    {
        Py_DECREF(type);
        return NULL;
    }
    return type;
}
