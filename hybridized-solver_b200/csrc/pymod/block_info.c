/*
 * block_info.c - `BlockInfo(row, col, val)`: an immutable (row, col, value) holder with
 * properties row, col, shape and value (the reference's src/block_info.c:3-104). No
 * other code uses it; it is kept for the API surface.
 */
#include "pymod.h"

#include <string.h>

typedef struct
{
    PyObject_VAR_HEAD uint64_t row;
    uint64_t col;
    uint64_t rows;
    uint64_t cols;
    double val[];
} block_info_object;

static PyObject *block_info_new(PyTypeObject *type, PyObject *args, PyObject *kwds)
{
    long row, col;
    PyObject *py_val;
    static char *kwlist[] = {"row", "col", "val", NULL};
    if (!PyArg_ParseTupleAndKeywords(args, kwds, "llO", kwlist, &row, &col, &py_val))
        return NULL;
    PyArrayObject *val =
        (PyArrayObject *)PyArray_FROMANY(py_val, NPY_DOUBLE, 2, 2, NPY_ARRAY_C_CONTIGUOUS | NPY_ARRAY_ALIGNED);
    if (!val)
        return NULL;
    const npy_intp total = PyArray_SIZE(val);
    block_info_object *self = (block_info_object *)type->tp_alloc(type, total);
    if (!self)
    {
        Py_DECREF(val);
        return NULL;
    }
    self->row = (uint64_t)row;
    self->col = (uint64_t)col;
    self->rows = (uint64_t)PyArray_DIM(val, 0);
    self->cols = (uint64_t)PyArray_DIM(val, 1);
    memcpy(self->val, PyArray_DATA(val), (size_t)total * sizeof(double));
    Py_DECREF(val);
    return (PyObject *)self;
}

static void block_info_dealloc(PyObject *self)
{
    PyTypeObject *tp = Py_TYPE(self);
    PyObject_GC_UnTrack(self);
    tp->tp_free(self);
    Py_DECREF(tp);
}

static PyObject *block_info_row(PyObject *self, void *Py_UNUSED(c))
{
    return PyLong_FromUnsignedLongLong(((block_info_object *)self)->row);
}

static PyObject *block_info_col(PyObject *self, void *Py_UNUSED(c))
{
    return PyLong_FromUnsignedLongLong(((block_info_object *)self)->col);
}

static PyObject *block_info_shape(PyObject *self, void *Py_UNUSED(c))
{
    const block_info_object *b = (block_info_object *)self;
    return Py_BuildValue("(nn)", (Py_ssize_t)b->rows, (Py_ssize_t)b->cols);
}

static PyObject *block_info_value(PyObject *self, void *Py_UNUSED(c))
{
    block_info_object *b = (block_info_object *)self;
    const npy_intp dims[2] = {(npy_intp)b->rows, (npy_intp)b->cols};
    PyArrayObject *arr = (PyArrayObject *)PyArray_SimpleNewFromData(2, dims, NPY_DOUBLE, b->val);
    if (!arr)
        return NULL;
    Py_INCREF(self);
    if (PyArray_SetBaseObject(arr, self) < 0)
    {
        Py_DECREF(arr);
        return NULL;
    }
    return (PyObject *)arr;
}

static PyGetSetDef block_info_getset[] = {
    {"row", block_info_row, NULL, "The row index of the block.", NULL},
    {"col", block_info_col, NULL, "The column index of the block.", NULL},
    {"shape", block_info_shape, NULL, "The shape of the block.", NULL},
    {"value", block_info_value, NULL, "The block value.", NULL},
    {NULL, NULL, NULL, NULL, NULL},
};

static PyType_Slot block_info_slots[] = {
    {Py_tp_new, block_info_new},
    {Py_tp_dealloc, block_info_dealloc},
    {Py_tp_getset, block_info_getset},
    {Py_tp_traverse, pymod_traverse_type},
    {Py_tp_doc, "BlockInfo(row: int, col: int, val: numpy.typing.ArrayLike)\nType describing a block.\n"},
    {0, NULL},
};

PyType_Spec pymod_block_info_spec = {
    .name = "hybsol._mod.BlockInfo",
    .basicsize = sizeof(block_info_object),
    .itemsize = sizeof(double),
    .flags = Py_TPFLAGS_DEFAULT | Py_TPFLAGS_HEAPTYPE | Py_TPFLAGS_HAVE_GC | Py_TPFLAGS_IMMUTABLETYPE,
    .slots = block_info_slots,
};
