/*
 * block_system.c - `hybsol._mod.BlockSystem`, the reference's BlockSystem type
 * (src/block_system.c:3-2216, typed at python/hybsol/_mod.pyi:29-356) rebuilt over the
 * B200 C ABI. Method names, keyword names, defaults, return values and exception types
 * follow the reference; deviations are listed in the method docstrings.
 *
 * State: before decompose() the blocks live in host rows (sorted {col, values} arrays)
 * so that assembly, reordering and the fine-grained row operations behave as in the
 * reference; every block product and factorisation those operations do runs on the GPU
 * through hyb_block_* entry points. decompose() uploads the pattern and values, factors
 * on the device and frees the host rows; the factors then stay on the device.
 */
#include "pymod.h"

#include <inttypes.h>
#include <stdlib.h>
#include <string.h>

typedef struct
{
    uint64_t col;
    double *vals;
} entry_t;

typedef struct
{
    uint64_t count;
    uint64_t capacity;
    entry_t *e; /* ascending col */
} hrow_t;

typedef struct
{
    PyObject_HEAD uint64_t n;
    uint64_t *offsets; /* n + 1 */
    hrow_t *rows;      /* host rows; NULL once decomposed */
    hyb_system *dev;   /* device system; non-NULL once decomposed */
    int precision;
    hyb_decompose_info dinfo;
    hyb_solve_info sinfo;
    int solve_status;
} bs_object;

/* ------------------------------------------------------------------------------- */
/* small helpers                                                                   */

static inline uint64_t bsize(const bs_object *s, uint64_t i)
{
    return s->offsets[i + 1] - s->offsets[i];
}

static uint64_t row_find_geq(const hrow_t *row, uint64_t col)
{
    uint64_t lo = 0, hi = row->count;
    while (lo < hi)
    {
        const uint64_t mid = lo + (hi - lo) / 2;
        if (row->e[mid].col < col)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

static entry_t *row_find(const hrow_t *row, uint64_t col)
{
    const uint64_t p = row_find_geq(row, col);
    return (p < row->count && row->e[p].col == col) ? row->e + p : NULL;
}

static int row_reserve(hrow_t *row, uint64_t need)
{
    if (row->capacity >= need)
        return 0;
    uint64_t cap = row->capacity ? row->capacity : 8;
    while (cap < need)
        cap *= 2;
    entry_t *p = (entry_t *)PyMem_RawRealloc(row->e, cap * sizeof(entry_t));
    if (!p)
        return -1;
    row->e = p;
    row->capacity = cap;
    return 0;
}

static void rows_free(hrow_t *rows, uint64_t n)
{
    if (!rows)
        return;
    for (uint64_t i = 0; i < n; ++i)
    {
        for (uint64_t j = 0; j < rows[i].count; ++j)
            PyMem_RawFree(rows[i].e[j].vals);
        PyMem_RawFree(rows[i].e);
    }
    PyMem_RawFree(rows);
}

static int raise_status(int status, const char *what)
{
    if (status == HYB_FAILED_ALLOC)
        PyErr_Format(PyExc_MemoryError, "%s: %s (%s)", what, hyb_status_string(status), hyb_last_cuda_error());
    else if (status == HYB_CUDA_ERROR || status == HYB_NO_DEVICE)
        PyErr_Format(PyExc_RuntimeError, "%s: %s (%s)", what, hyb_status_string(status), hyb_last_cuda_error());
    else
        PyErr_Format(PyExc_RuntimeError, "%s: %s", what, hyb_status_string(status));
    return -1;
}

static int check_index(uint64_t n, Py_ssize_t idx, const char *name)
{
    if (idx < 0 || (uint64_t)idx >= n)
    {
        PyErr_Format(PyExc_ValueError, "%s must be in the range [0, %" PRIu64 "), but it was %zd.", name, n, idx);
        return -1;
    }
    return 0;
}

static int ensure_not_decomposed(const bs_object *s)
{
    if (s->dev)
    {
        PyErr_SetString(PyExc_RuntimeError, "The system has already been decomposed.");
        return -1;
    }
    return 0;
}

static int ensure_decomposed(const bs_object *s)
{
    if (!s->dev)
    {
        PyErr_SetString(PyExc_RuntimeError, "The system has not been decomposed yet.");
        return -1;
    }
    return 0;
}

/* Fastcall argument parsing: positional then keyword, optional args keep their value. */
typedef enum
{
    ARG_END = 0,
    ARG_SSIZE,
    ARG_OBJECT,
    ARG_DOUBLE,
} argkind_t;

typedef struct
{
    argkind_t kind;
    const char *name;
    void *out;
    int optional;
    int kwonly;
} argspec_t;

static int parse_args(PyObject *const *args, Py_ssize_t nargs, PyObject *kwnames, const argspec_t *spec)
{
    enum
    {
        MAXA = 8
    };
    Py_ssize_t count = 0, npos = 0;
    while (spec[count].kind != ARG_END)
    {
        if (!spec[count].kwonly)
            npos = count + 1;
        ++count;
    }
    if (nargs > npos)
    {
        PyErr_Format(PyExc_TypeError, "Expected at most %zd positional arguments, got %zd.", npos, nargs);
        return -1;
    }
    PyObject *given[MAXA] = {0};
    for (Py_ssize_t i = 0; i < nargs; ++i)
        given[i] = args[i];
    const Py_ssize_t nkw = kwnames ? PyTuple_GET_SIZE(kwnames) : 0;
    for (Py_ssize_t k = 0; k < nkw; ++k)
    {
        const char *kw = PyUnicode_AsUTF8(PyTuple_GET_ITEM(kwnames, k));
        if (!kw)
            return -1;
        Py_ssize_t i = 0;
        while (i < count && strcmp(kw, spec[i].name) != 0)
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
        PyObject *v = given[i];
        if (!v)
        {
            if (spec[i].optional)
                continue;
            PyErr_Format(PyExc_TypeError, "Missing required argument '%s'.", spec[i].name);
            return -1;
        }
        switch (spec[i].kind)
        {
        case ARG_SSIZE: {
            const Py_ssize_t x = PyNumber_AsSsize_t(v, PyExc_OverflowError);
            if (x == -1 && PyErr_Occurred())
                return -1;
            *(Py_ssize_t *)spec[i].out = x;
            break;
        }
        case ARG_DOUBLE: {
            const double x = PyFloat_AsDouble(v);
            if (x == -1.0 && PyErr_Occurred())
                return -1;
            *(double *)spec[i].out = x;
            break;
        }
        case ARG_OBJECT:
            *(PyObject **)spec[i].out = (spec[i].optional && v == Py_None) ? NULL : v;
            break;
        default:
            return -1;
        }
    }
    return 0;
}

static int no_args(Py_ssize_t nargs, PyObject *kwnames, const char *msg)
{
    if (nargs != 0 || (kwnames && PyTuple_GET_SIZE(kwnames) != 0))
    {
        PyErr_SetString(PyExc_TypeError, msg);
        return -1;
    }
    return 0;
}

/* A 2-D float64 C-contiguous copy-or-view of `obj` with the given shape. */
static PyArrayObject *as_block(PyObject *obj, uint64_t rows, uint64_t cols, const char *name)
{
    PyArrayObject *arr =
        (PyArrayObject *)PyArray_FROMANY(obj, NPY_DOUBLE, 2, 2, NPY_ARRAY_C_CONTIGUOUS | NPY_ARRAY_ALIGNED);
    if (!arr)
        return NULL;
    if ((uint64_t)PyArray_DIM(arr, 0) != rows || (uint64_t)PyArray_DIM(arr, 1) != cols)
    {
        PyErr_Format(PyExc_ValueError, "Array %s has shape (%zd, %zd), expected (%" PRIu64 ", %" PRIu64 ").", name,
                     (Py_ssize_t)PyArray_DIM(arr, 0), (Py_ssize_t)PyArray_DIM(arr, 1), rows, cols);
        Py_DECREF(arr);
        return NULL;
    }
    return arr;
}

/* Checks a caller-provided output array against dtype, flags and shape. */
static int check_out(PyArrayObject *out, int ndim, const npy_intp *dims, const char *name)
{
    if (PyArray_TYPE(out) != NPY_DOUBLE ||
        !PyArray_CHKFLAGS(out, NPY_ARRAY_C_CONTIGUOUS | NPY_ARRAY_ALIGNED | NPY_ARRAY_WRITEABLE))
    {
        PyErr_Format(PyExc_ValueError, "Array %s must be a writeable, aligned, C-contiguous float64 array.", name);
        return -1;
    }
    if (PyArray_NDIM(out) != ndim)
    {
        PyErr_Format(PyExc_ValueError, "Array %s has %d dimensions, expected %d.", name, PyArray_NDIM(out), ndim);
        return -1;
    }
    for (int i = 0; i < ndim; ++i)
        if (PyArray_DIM(out, i) != dims[i])
        {
            PyErr_Format(PyExc_ValueError, "Array %s has the wrong shape.", name);
            return -1;
        }
    return 0;
}

static bs_object *check_self(PyObject *self, PyTypeObject *defining_class)
{
    const pymod_state *st = pymod_state_of(defining_class ? defining_class : Py_TYPE(self));
    if (!st)
        return NULL;
    if (!PyObject_TypeCheck(self, st->type_block_system))
    {
        PyErr_Format(PyExc_TypeError, "Expected a hybsol._mod.BlockSystem, got a %s.", Py_TYPE(self)->tp_name);
        return NULL;
    }
    return (bs_object *)self;
}

/* Row columns of the current pattern (host rows, or the device's filled pattern). */
static PyObject *row_cols_tuple(const bs_object *s, uint64_t r)
{
    if (!s->dev)
    {
        const hrow_t *row = s->rows + r;
        PyObject *t = PyTuple_New((Py_ssize_t)row->count);
        if (!t)
            return NULL;
        for (uint64_t j = 0; j < row->count; ++j)
        {
            PyObject *v = PyLong_FromUnsignedLongLong(row->e[j].col);
            if (!v)
            {
                Py_DECREF(t);
                return NULL;
            }
            PyTuple_SET_ITEM(t, (Py_ssize_t)j, v);
        }
        return t;
    }
    uint64_t cnt = 0;
    int st = hyb_row_count(s->dev, r, &cnt);
    if (st)
        return raise_status(st, "hyb_row_count"), NULL;
    uint64_t *cols = (uint64_t *)PyMem_Malloc((cnt + 1) * sizeof(uint64_t));
    if (!cols)
        return PyErr_NoMemory();
    st = hyb_row_cols(s->dev, r, cols);
    if (st)
    {
        PyMem_Free(cols);
        return raise_status(st, "hyb_row_cols"), NULL;
    }
    PyObject *t = PyTuple_New((Py_ssize_t)cnt);
    for (uint64_t j = 0; t && j < cnt; ++j)
    {
        PyObject *v = PyLong_FromUnsignedLongLong(cols[j]);
        if (!v)
        {
            Py_CLEAR(t);
            break;
        }
        PyTuple_SET_ITEM(t, (Py_ssize_t)j, v);
    }
    PyMem_Free(cols);
    return t;
}

/* Column list of a row into a freshly allocated array (caller frees with PyMem_Free). */
static int row_cols_array(const bs_object *s, uint64_t r, uint64_t **out, uint64_t *count)
{
    if (!s->dev)
    {
        const hrow_t *row = s->rows + r;
        *count = row->count;
        *out = (uint64_t *)PyMem_Malloc((row->count + 1) * sizeof(uint64_t));
        if (!*out)
            return PyErr_NoMemory(), -1;
        for (uint64_t j = 0; j < row->count; ++j)
            (*out)[j] = row->e[j].col;
        return 0;
    }
    int st = hyb_row_count(s->dev, r, count);
    if (st)
        return raise_status(st, "hyb_row_count");
    *out = (uint64_t *)PyMem_Malloc((*count + 1) * sizeof(uint64_t));
    if (!*out)
        return PyErr_NoMemory(), -1;
    st = hyb_row_cols(s->dev, r, *out);
    if (st)
    {
        PyMem_Free(*out);
        return raise_status(st, "hyb_row_cols");
    }
    return 0;
}

/* Copies block (r, c) into `out`; returns 1 if absent, -1 on error. */
static int read_block(const bs_object *s, uint64_t r, uint64_t c, double *out)
{
    if (!s->dev)
    {
        const entry_t *e = row_find(s->rows + r, c);
        if (!e)
            return 1;
        memcpy(out, e->vals, bsize(s, r) * bsize(s, c) * sizeof(double));
        return 0;
    }
    const int st = hyb_get_block(s->dev, r, c, out);
    if (st == HYB_BLOCK_NOT_IN_SYSTEM)
        return 1;
    if (st)
        return raise_status(st, "hyb_get_block");
    return 0;
}

/* ------------------------------------------------------------------------------- */
/* construction / destruction                                                      */

static PyObject *bs_new(PyTypeObject *type, PyObject *args, PyObject *kwds)
{
    if (kwds && PyDict_GET_SIZE(kwds) != 0)
    {
        PyErr_SetString(PyExc_TypeError, "BlockSystem takes no keyword arguments");
        return NULL;
    }
    const Py_ssize_t n = PyTuple_GET_SIZE(args);
    if (n == 0)
    {
        PyErr_SetString(PyExc_ValueError, "BlockSystem requires at least one block");
        return NULL;
    }
    bs_object *self = (bs_object *)type->tp_alloc(type, 0);
    if (!self)
        return NULL;
    self->n = (uint64_t)n;
    self->offsets = (uint64_t *)PyMem_Malloc(((size_t)n + 1) * sizeof(uint64_t));
    self->rows = (hrow_t *)PyMem_RawCalloc((size_t)n, sizeof(hrow_t));
    if (!self->offsets || !self->rows)
    {
        Py_DECREF(self);
        return PyErr_NoMemory();
    }
    self->offsets[0] = 0;
    for (Py_ssize_t i = 0; i < n; ++i)
    {
        const Py_ssize_t sz = PyNumber_AsSsize_t(PyTuple_GET_ITEM(args, i), PyExc_ValueError);
        if (sz == -1 && PyErr_Occurred())
        {
            Py_DECREF(self);
            return NULL;
        }
        if (sz <= 0)
        {
            PyErr_Format(PyExc_ValueError, "Block size of block %zd is %zd.", i, sz);
            Py_DECREF(self);
            return NULL;
        }
        self->offsets[i + 1] = self->offsets[i] + (uint64_t)sz;
    }
    return (PyObject *)self;
}

static void bs_dealloc(PyObject *obj)
{
    bs_object *self = (bs_object *)obj;
    PyTypeObject *tp = Py_TYPE(obj);
    PyObject_GC_UnTrack(obj);
    rows_free(self->rows, self->n);
    self->rows = NULL;
    if (self->dev)
    {
        Py_BEGIN_ALLOW_THREADS;
        hyb_system_destroy(self->dev);
        Py_END_ALLOW_THREADS;
        self->dev = NULL;
    }
    PyMem_Free(self->offsets);
    self->offsets = NULL;
    tp->tp_free(obj);
    Py_DECREF(tp);
}

/* ------------------------------------------------------------------------------- */
/* assembly and accessors                                                          */

/* Adds block (r, c) with row-major values `src` to the host rows: summed into a block already
 * present (block_system_add_block, src/blocks.c:36-45), else inserted in column order.
 * Returns -1 with RuntimeError set when memory runs out. */
static int host_add(bs_object *s, uint64_t r, uint64_t c, const double *src)
{
    const uint64_t nv = bsize(s, r) * bsize(s, c);
    hrow_t *row = s->rows + r;
    const uint64_t p = row_find_geq(row, c);
    if (p < row->count && row->e[p].col == c)
    {
        double *dst = row->e[p].vals;
        for (uint64_t i = 0; i < nv; ++i)
            dst[i] += src[i];
        return 0;
    }
    double *vals = (double *)PyMem_RawMalloc(nv * sizeof(double));
    if (!vals || row_reserve(row, row->count + 1) < 0)
    {
        PyMem_RawFree(vals);
        PyErr_SetString(PyExc_RuntimeError, "Failed to add block to block system.");
        return -1;
    }
    memcpy(vals, src, nv * sizeof(double));
    memmove(row->e + p + 1, row->e + p, (row->count - p) * sizeof(entry_t));
    row->e[p].col = c;
    row->e[p].vals = vals;
    row->count += 1;
    return 0;
}

static PyObject *bs_add_block(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                              PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s || ensure_not_decomposed(s) < 0)
        return NULL;
    Py_ssize_t r, c;
    PyObject *val;
    const argspec_t spec[] = {{ARG_SSIZE, "row", &r, 0, 0}, {ARG_SSIZE, "col", &c, 0, 0}, {ARG_OBJECT, "val", &val, 0, 0}, {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0)
        return NULL;
    if (check_index(s->n, r, "Row index") < 0 || check_index(s->n, c, "Column index") < 0)
        return NULL;
    PyArrayObject *arr = as_block(val, bsize(s, r), bsize(s, c), "val");
    if (!arr)
        return NULL;
    const int rc = host_add(s, (uint64_t)r, (uint64_t)c, (const double *)PyArray_DATA(arr));
    Py_DECREF(arr);
    if (rc < 0)
        return NULL;
    Py_RETURN_NONE;
}

/* A 1-D int64 C-contiguous array from an integer array-like. */
static PyArrayObject *as_index_array(PyObject *obj, const char *name)
{
    PyArrayObject *a = (PyArrayObject *)PyArray_FROM_O(obj);
    if (!a)
        return NULL;
    if (PyArray_NDIM(a) != 1 || (!PyArray_ISINTEGER(a) && PyArray_SIZE(a) != 0))
    {
        PyErr_Format(PyExc_ValueError, "Array %s must be a 1-D array of integers.", name);
        Py_DECREF(a);
        return NULL;
    }
    PyArrayObject *out = (PyArrayObject *)PyArray_FROMANY((PyObject *)a, NPY_INT64, 1, 1,
                                                          NPY_ARRAY_C_CONTIGUOUS | NPY_ARRAY_ALIGNED | NPY_ARRAY_FORCECAST);
    Py_DECREF(a);
    return out;
}

/* Bulk form of add_block (no counterpart in the reference): block i is (rows[i], cols[i])
 * with its row-major values next in the 1-D `values`. Everything is checked before the
 * first block is added; blocks are then added in order, so repeated positions are summed
 * exactly as by successive add_block calls. */
static PyObject *bs_add_blocks(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                               PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s || ensure_not_decomposed(s) < 0)
        return NULL;
    PyObject *orows, *ocols, *ovals;
    const argspec_t spec[] = {{ARG_OBJECT, "rows", &orows, 0, 0},
                              {ARG_OBJECT, "cols", &ocols, 0, 0},
                              {ARG_OBJECT, "values", &ovals, 0, 0},
                              {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0)
        return NULL;
    PyArrayObject *ar = as_index_array(orows, "rows");
    PyArrayObject *ac = ar ? as_index_array(ocols, "cols") : NULL;
    PyArrayObject *av =
        ac ? (PyArrayObject *)PyArray_FROMANY(ovals, NPY_DOUBLE, 1, 1, NPY_ARRAY_C_CONTIGUOUS | NPY_ARRAY_ALIGNED) : NULL;
    PyObject *result = NULL;
    if (!av)
        goto done;
    const npy_intp nb = PyArray_DIM(ar, 0);
    if (PyArray_DIM(ac, 0) != nb)
    {
        PyErr_Format(PyExc_ValueError, "Arrays rows and cols have %zd and %zd entries.", (Py_ssize_t)nb,
                     (Py_ssize_t)PyArray_DIM(ac, 0));
        goto done;
    }
    const int64_t *rr = (const int64_t *)PyArray_DATA(ar), *cc = (const int64_t *)PyArray_DATA(ac);
    uint64_t total = 0;
    for (npy_intp i = 0; i < nb; ++i)
    {
        if (check_index(s->n, (Py_ssize_t)rr[i], "Row index") < 0 || check_index(s->n, (Py_ssize_t)cc[i], "Column index") < 0)
            goto done;
        total += bsize(s, (uint64_t)rr[i]) * bsize(s, (uint64_t)cc[i]);
    }
    if ((uint64_t)PyArray_DIM(av, 0) != total)
    {
        PyErr_Format(PyExc_ValueError, "Array values has %zd entries, the blocks need %" PRIu64 ".",
                     (Py_ssize_t)PyArray_DIM(av, 0), total);
        goto done;
    }
    const double *v = (const double *)PyArray_DATA(av);
    for (npy_intp i = 0; i < nb; ++i)
    {
        const uint64_t r = (uint64_t)rr[i], c = (uint64_t)cc[i];
        if (host_add(s, r, c, v) < 0)
            goto done;
        v += bsize(s, r) * bsize(s, c);
    }
    result = Py_None;
    Py_INCREF(result);
done:
    Py_XDECREF(ar);
    Py_XDECREF(ac);
    Py_XDECREF(av);
    return result;
}

static PyObject *bs_is_valid(PyObject *self, PyTypeObject *cls, PyObject *const *Py_UNUSED(args), Py_ssize_t nargs,
                             PyObject *kwnames)
{
    if (no_args(nargs, kwnames, "BlockSystem.is_valid() takes no arguments.") < 0)
        return NULL;
    bs_object *s = check_self(self, cls);
    if (!s)
        return NULL;
    /* block_system_is_valid (src/blocks.c:77-110): every row must reach its diagonal, and
     * each block left of it must have its transpose partner. */
    for (uint64_t i = 0; i < s->n; ++i)
    {
        uint64_t *cols, cnt;
        if (row_cols_array(s, i, &cols, &cnt) < 0)
            return NULL;
        int ok = 1;
        for (uint64_t j = 0; j < cnt && ok; ++j)
        {
            const uint64_t c = cols[j];
            if (c == i)
                break;
            if (c > i)
            {
                ok = 0;
                break;
            }
            uint64_t *oc, ocnt;
            if (row_cols_array(s, c, &oc, &ocnt) < 0)
            {
                PyMem_Free(cols);
                return NULL;
            }
            int found = 0;
            for (uint64_t q = 0; q < ocnt; ++q)
                found |= oc[q] == i;
            PyMem_Free(oc);
            ok = found;
        }
        PyMem_Free(cols);
        if (!ok)
            Py_RETURN_FALSE;
    }
    Py_RETURN_TRUE;
}

static PyObject *bs_as_array(PyObject *self, PyTypeObject *cls, PyObject *const *Py_UNUSED(args), Py_ssize_t nargs,
                             PyObject *kwnames)
{
    if (no_args(nargs, kwnames, "BlockSystem.as_array() takes no arguments.") < 0)
        return NULL;
    bs_object *s = check_self(self, cls);
    if (!s)
        return NULL;
    const uint64_t dof = s->offsets[s->n];
    const npy_intp dims[2] = {(npy_intp)dof, (npy_intp)dof};
    PyArrayObject *arr = (PyArrayObject *)PyArray_ZEROS(2, dims, NPY_DOUBLE, 0);
    if (!arr)
        return NULL;
    double *a = (double *)PyArray_DATA(arr);
    uint64_t max_size = 0;
    for (uint64_t i = 0; i < s->n; ++i)
        max_size = bsize(s, i) > max_size ? bsize(s, i) : max_size;
    double *buf = (double *)PyMem_Malloc(max_size * max_size * sizeof(double) + 8);
    if (!buf)
    {
        Py_DECREF(arr);
        return PyErr_NoMemory();
    }
    for (uint64_t i = 0; i < s->n; ++i)
    {
        uint64_t *cols, cnt;
        if (row_cols_array(s, i, &cols, &cnt) < 0)
            goto fail;
        for (uint64_t j = 0; j < cnt; ++j)
        {
            const uint64_t c = cols[j], nr = bsize(s, i), nc = bsize(s, c);
            if (read_block(s, i, c, buf) < 0)
            {
                PyMem_Free(cols);
                goto fail;
            }
            for (uint64_t q = 0; q < nr; ++q)
                memcpy(a + (s->offsets[i] + q) * dof + s->offsets[c], buf + q * nc, nc * sizeof(double));
        }
        PyMem_Free(cols);
    }
    PyMem_Free(buf);
    return (PyObject *)arr;
fail:
    PyMem_Free(buf);
    Py_DECREF(arr);
    return NULL;
}

static PyObject *bs_get_row_block_indices(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                                          PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s)
        return NULL;
    Py_ssize_t r;
    const argspec_t spec[] = {{ARG_SSIZE, "row", &r, 0, 0}, {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0 || check_index(s->n, r, "Row index") < 0)
        return NULL;
    return row_cols_tuple(s, (uint64_t)r);
}

static PyObject *bs_get_block(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                              PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s)
        return NULL;
    Py_ssize_t r, c;
    const argspec_t spec[] = {{ARG_SSIZE, "row", &r, 0, 0}, {ARG_SSIZE, "col", &c, 0, 0}, {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0 || check_index(s->n, r, "Row index") < 0 ||
        check_index(s->n, c, "Col index") < 0)
        return NULL;
    const npy_intp dims[2] = {(npy_intp)bsize(s, r), (npy_intp)bsize(s, c)};
    PyArrayObject *arr = (PyArrayObject *)PyArray_SimpleNew(2, dims, NPY_DOUBLE);
    if (!arr)
        return NULL;
    const int rc = read_block(s, (uint64_t)r, (uint64_t)c, (double *)PyArray_DATA(arr));
    if (rc != 0)
    {
        Py_DECREF(arr);
        if (rc > 0)
            PyErr_Format(PyExc_ValueError, "The system does not contain the block (%zd, %zd).", r, c);
        return NULL;
    }
    return (PyObject *)arr;
}

static PyObject *bs_get_block_size(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                                   PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s)
        return NULL;
    Py_ssize_t r, c;
    const argspec_t spec[] = {{ARG_SSIZE, "row", &r, 0, 0}, {ARG_SSIZE, "col", &c, 0, 0}, {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0 || check_index(s->n, r, "Row index") < 0 ||
        check_index(s->n, c, "Col index") < 0)
        return NULL;
    return Py_BuildValue("(nn)", (Py_ssize_t)bsize(s, r), (Py_ssize_t)bsize(s, c));
}

static PyObject *bs_has_block(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                              PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s)
        return NULL;
    Py_ssize_t r, c;
    const argspec_t spec[] = {{ARG_SSIZE, "row", &r, 0, 0}, {ARG_SSIZE, "col", &c, 0, 0}, {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0 || check_index(s->n, r, "Row index") < 0 ||
        check_index(s->n, c, "Column index") < 0)
        return NULL;
    uint64_t *cols, cnt;
    if (row_cols_array(s, (uint64_t)r, &cols, &cnt) < 0)
        return NULL;
    int found = 0;
    for (uint64_t j = 0; j < cnt; ++j)
        found |= cols[j] == (uint64_t)c;
    PyMem_Free(cols);
    return PyBool_FromLong(found);
}

static PyObject *bs_no_lower_connections(PyObject *self, PyTypeObject *cls, PyObject *const *Py_UNUSED(args),
                                         Py_ssize_t nargs, PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s || no_args(nargs, kwnames, "No arguments accepted.") < 0)
        return NULL;
    const npy_intp dim = (npy_intp)s->n;
    PyArrayObject *arr = (PyArrayObject *)PyArray_SimpleNew(1, &dim, NPY_BOOL);
    if (!arr)
        return NULL;
    npy_bool *out = (npy_bool *)PyArray_DATA(arr);
    for (uint64_t i = 0; i < s->n; ++i)
    {
        uint64_t *cols, cnt;
        if (row_cols_array(s, i, &cols, &cnt) < 0)
        {
            Py_DECREF(arr);
            return NULL;
        }
        out[i] = cnt == 0 ? 1 : cols[0] >= i;
        PyMem_Free(cols);
    }
    return (PyObject *)arr;
}

static PyObject *bs_first_column(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                                 PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s)
        return NULL;
    Py_ssize_t r;
    const argspec_t spec[] = {{ARG_SSIZE, "row", &r, 0, 0}, {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0 || check_index(s->n, r, "Row index") < 0)
        return NULL;
    uint64_t *cols, cnt;
    if (row_cols_array(s, (uint64_t)r, &cols, &cnt) < 0)
        return NULL;
    if (cnt == 0)
    {
        PyMem_Free(cols);
        PyErr_SetString(PyExc_ValueError, "Row has no entries.");
        return NULL;
    }
    PyObject *v = PyLong_FromUnsignedLongLong(cols[0]);
    PyMem_Free(cols);
    return v;
}

static PyObject *bs_get_next_column_index(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                                          PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s)
        return NULL;
    Py_ssize_t r, c;
    const argspec_t spec[] = {{ARG_SSIZE, "row", &r, 0, 0}, {ARG_SSIZE, "col", &c, 0, 0}, {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0 || check_index(s->n, r, "Row index") < 0 ||
        check_index(s->n, c, "Column index") < 0)
        return NULL;
    uint64_t *cols, cnt;
    if (row_cols_array(s, (uint64_t)r, &cols, &cnt) < 0)
        return NULL;
    if (cnt == 0)
    {
        PyMem_Free(cols);
        PyErr_SetString(PyExc_ValueError, "Row has no entries.");
        return NULL;
    }
    uint64_t j = 0;
    while (j < cnt && cols[j] < (uint64_t)c + 1)
        ++j;
    if (j == cnt)
    {
        PyMem_Free(cols);
        PyErr_SetString(PyExc_ValueError, "Row has no entries after column index.");
        return NULL;
    }
    PyObject *v = PyLong_FromUnsignedLongLong(cols[j]);
    PyMem_Free(cols);
    return v;
}

/* ------------------------------------------------------------------------------- */
/* fine-grained row operations (host storage, GPU arithmetic)                      */

static PyObject *bs_multiply_row(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                                 PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s || ensure_not_decomposed(s) < 0)
        return NULL;
    Py_ssize_t r, start = 0;
    PyObject *val;
    const argspec_t spec[] = {
        {ARG_SSIZE, "row", &r, 0, 0}, {ARG_OBJECT, "val", &val, 0, 0}, {ARG_SSIZE, "start", &start, 1, 0}, {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0)
        return NULL;
    if (check_index(s->n, r, "Row index") < 0 || check_index(s->n, start, "Start index") < 0)
        return NULL;
    PyArrayObject *arr =
        (PyArrayObject *)PyArray_FROMANY(val, NPY_DOUBLE, 2, 2, NPY_ARRAY_C_CONTIGUOUS | NPY_ARRAY_ALIGNED);
    if (!arr)
        return NULL;
    const uint64_t m = bsize(s, r);
    if ((uint64_t)PyArray_DIM(arr, 0) != m || (uint64_t)PyArray_DIM(arr, 1) != m)
    {
        PyErr_Format(PyExc_ValueError, "Value must be a square matrix of size %zd.", (Py_ssize_t)m);
        Py_DECREF(arr);
        return NULL;
    }
    /* Each block at or after `start` becomes val @ block (src/block_system.c:454-538). */
    hrow_t *row = s->rows + r;
    int st = HYB_SUCCESS;
    for (uint64_t j = 0; j < row->count && st == HYB_SUCCESS; ++j)
    {
        if (row->e[j].col < (uint64_t)start)
            continue;
        const uint64_t nc = bsize(s, row->e[j].col);
        double *tmp = (double *)PyMem_RawMalloc(m * nc * sizeof(double));
        if (!tmp)
        {
            Py_DECREF(arr);
            return PyErr_NoMemory();
        }
        Py_BEGIN_ALLOW_THREADS;
        st = hyb_block_gemm(m, m, nc, (const double *)PyArray_DATA(arr), row->e[j].vals, tmp, 0, HYB_MEMORY_HOST);
        Py_END_ALLOW_THREADS;
        if (st == HYB_SUCCESS)
            memcpy(row->e[j].vals, tmp, m * nc * sizeof(double));
        PyMem_RawFree(tmp);
    }
    Py_DECREF(arr);
    if (st)
        return raise_status(st, "multiply_row"), NULL;
    Py_RETURN_NONE;
}

static PyObject *bs_eliminate_row(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                                  PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s || ensure_not_decomposed(s) < 0)
        return NULL;
    Py_ssize_t isrc, itgt;
    PyObject *val;
    const argspec_t spec[] = {
        {ARG_SSIZE, "row_src", &isrc, 0, 0}, {ARG_SSIZE, "row_tgt", &itgt, 0, 0}, {ARG_OBJECT, "val", &val, 0, 0}, {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0)
        return NULL;
    if (check_index(s->n, isrc, "Row index source") < 0 || check_index(s->n, itgt, "Row index target") < 0)
        return NULL;
    const uint64_t src = (uint64_t)isrc, tgt = (uint64_t)itgt;
    hrow_t *rt = s->rows + tgt;
    const hrow_t *rs = s->rows + src;
    /* The reference requires one of the two rows to carry column `src` where its walk
     * stops (src/block_system.c:621-626). */
    if (!row_find(rt, src) && !row_find(rs, src))
    {
        PyErr_Format(PyExc_ValueError,
                     "Source and target blocks must both contain the diagonal block for the row %" PRIu64 ".", src);
        return NULL;
    }
    const uint64_t mt = bsize(s, tgt), ms = bsize(s, src);
    PyArrayObject *arr = as_block(val, mt, ms, "val");
    if (!arr)
        return NULL;
    const double *mult = (const double *)PyArray_DATA(arr);
    /* Columns > src: T[c] -= S * R[c] where T has c, new fill T[c] = -(S * R[c]) where it
     * has not (block_system_eliminate_row, src/block_system.c:552-766). */
    const uint64_t ps = row_find_geq(rs, src + 1), pt = row_find_geq(rt, src + 1);
    uint64_t extra = 0;
    for (uint64_t j = ps; j < rs->count; ++j)
        extra += row_find(rt, rs->e[j].col) == NULL;
    if (row_reserve(rt, rt->count + extra) < 0)
    {
        Py_DECREF(arr);
        return PyErr_NoMemory();
    }
    uint64_t a = rt->count, b = rs->count, k = rt->count + extra;
    int st = HYB_SUCCESS;
    /* Merge the columns first (existing target blocks or zeroed fill blocks), collecting the
     * products; then one batched device call applies them all. */
    const uint64_t nprod = rs->count - ps;
    const double **bsrc = (const double **)PyMem_RawMalloc((nprod ? nprod : 1) * sizeof(double *));
    double **cdst = (double **)PyMem_RawMalloc((nprod ? nprod : 1) * sizeof(double *));
    uint64_t *ncol = (uint64_t *)PyMem_RawMalloc((nprod ? nprod : 1) * sizeof(uint64_t));
    uint64_t np = 0;
    if (!bsrc || !cdst || !ncol)
        st = HYB_FAILED_ALLOC;
    while (b > ps && st == HYB_SUCCESS)
    {
        const entry_t *es = rs->e + (b - 1);
        if (a > pt && rt->e[a - 1].col > es->col)
        {
            rt->e[--k] = rt->e[--a];
            continue;
        }
        const uint64_t nc = bsize(s, es->col);
        if (a > pt && rt->e[a - 1].col == es->col)
        {
            entry_t e = rt->e[--a];
            rt->e[--k] = e;
        }
        else
        {
            double *fill = (double *)PyMem_RawCalloc(mt * nc, sizeof(double));
            if (!fill)
            {
                st = HYB_FAILED_ALLOC;
                break;
            }
            rt->e[--k].col = es->col;
            rt->e[k].vals = fill;
        }
        bsrc[np] = es->vals;
        cdst[np] = rt->e[k].vals;
        ncol[np] = nc;
        ++np;
        --b;
    }
    if (st == HYB_SUCCESS && np > 0)
    {
        Py_BEGIN_ALLOW_THREADS;
        st = hyb_block_gemm_batched(np, mt, ms, ncol, mult, bsrc, cdst, 1, HYB_MEMORY_HOST);
        Py_END_ALLOW_THREADS;
    }
    PyMem_RawFree((void *)bsrc);
    PyMem_RawFree(cdst);
    PyMem_RawFree(ncol);
    Py_DECREF(arr);
    if (st != HYB_SUCCESS)
    {
        /* As in the reference (src/block_system.c:714-731) the target row cannot be
         * recovered once the merge fails part-way; it is emptied. The live entries are the
         * unmoved prefix [0, a) and the merged suffix [k, count + extra). */
        for (uint64_t j = 0; j < a; ++j)
            PyMem_RawFree(rt->e[j].vals);
        for (uint64_t j = k; j < rt->count + extra; ++j)
            PyMem_RawFree(rt->e[j].vals);
        rt->count = 0;
        PyErr_Format(PyExc_MemoryError,
                     "Eliminating row %" PRIu64 " from row %" PRIu64 " failed (%s); the target row was erased.", src,
                     tgt, hyb_status_string(st));
        return NULL;
    }
    rt->count += extra;
    Py_RETURN_NONE;
}

static PyObject *bs_decompose_diagonal(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                                       PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s || ensure_not_decomposed(s) < 0)
        return NULL;
    Py_ssize_t i;
    const argspec_t spec[] = {{ARG_SSIZE, "idx", &i, 0, 0}, {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0 || check_index(s->n, i, "Block index") < 0)
        return NULL;
    entry_t *e = row_find(s->rows + i, (uint64_t)i);
    if (!e)
    {
        PyErr_Format(PyExc_ValueError, "Row %zd has no diagonal entry.", i);
        return NULL;
    }
    int st;
    Py_BEGIN_ALLOW_THREADS;
    st = hyb_block_lu(bsize(s, i), e->vals, HYB_MEMORY_HOST);
    Py_END_ALLOW_THREADS;
    if (st)
        return raise_status(st, "decompose_diagonal"), NULL;
    Py_RETURN_NONE;
}

static PyObject *bs_solve_diagonal(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                                   PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s)
        return NULL;
    Py_ssize_t i;
    PyObject *val, *out_obj = NULL;
    const argspec_t spec[] = {
        {ARG_SSIZE, "idx", &i, 0, 0}, {ARG_OBJECT, "val", &val, 0, 0}, {ARG_OBJECT, "out", &out_obj, 1, 0}, {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0 || check_index(s->n, i, "Block index") < 0)
        return NULL;
    if (out_obj && !PyArray_Check(out_obj))
    {
        PyErr_SetString(PyExc_TypeError, "Argument 'out' must be of type numpy.ndarray.");
        return NULL;
    }
    const uint64_t m = bsize(s, i);
    double *lu = (double *)PyMem_Malloc(m * m * sizeof(double));
    if (!lu)
        return PyErr_NoMemory();
    const int rc = read_block(s, (uint64_t)i, (uint64_t)i, lu);
    if (rc != 0)
    {
        PyMem_Free(lu);
        if (rc > 0)
            PyErr_Format(PyExc_ValueError, "Row %zd has no diagonal entry.", i);
        return NULL;
    }
    PyArrayObject *arr =
        (PyArrayObject *)PyArray_FROMANY(val, NPY_DOUBLE, 1, 2, NPY_ARRAY_C_CONTIGUOUS | NPY_ARRAY_ALIGNED);
    if (!arr)
    {
        PyMem_Free(lu);
        return NULL;
    }
    if ((uint64_t)PyArray_DIM(arr, 0) != m)
    {
        PyErr_Format(PyExc_ValueError, "Array val must have %" PRIu64 " rows.", m);
        goto fail;
    }
    PyArrayObject *out = (PyArrayObject *)out_obj;
    if (out)
    {
        if (check_out(out, PyArray_NDIM(arr), PyArray_DIMS(arr), "out") < 0)
            goto fail;
        Py_INCREF(out);
    }
    else
    {
        out = (PyArrayObject *)PyArray_SimpleNew(PyArray_NDIM(arr), PyArray_DIMS(arr), NPY_DOUBLE);
        if (!out)
            goto fail;
    }
    const uint64_t ncols = PyArray_NDIM(arr) == 2 ? (uint64_t)PyArray_DIM(arr, 1) : 1;
    int st;
    Py_BEGIN_ALLOW_THREADS;
    st = hyb_block_lu_solve(m, lu, ncols, (const double *)PyArray_DATA(arr), (double *)PyArray_DATA(out),
                            HYB_MEMORY_HOST);
    Py_END_ALLOW_THREADS;
    PyMem_Free(lu);
    Py_DECREF(arr);
    if (st)
    {
        Py_DECREF(out);
        return raise_status(st, "solve_diagonal"), NULL;
    }
    /* The reference returns None here (src/block_system.c:1055) although its stub promises
     * the output array; the array is returned, which callers ignoring the result don't see. */
    return (PyObject *)out;
fail:
    PyMem_Free(lu);
    Py_DECREF(arr);
    return NULL;
}

static PyObject *bs_row_apply_decomposition(PyObject *self, PyTypeObject *cls, PyObject *const *args,
                                            Py_ssize_t nargs, PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s)
        return NULL;
    Py_ssize_t r;
    const argspec_t spec[] = {{ARG_SSIZE, "row", &r, 0, 0}, {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0 || check_index(s->n, r, "Row index") < 0)
        return NULL;
    if (ensure_not_decomposed(s) < 0)
        return NULL;
    hrow_t *row = s->rows + r;
    if (row->count == 0)
    {
        PyErr_Format(PyExc_ValueError, "Row %zd has no entries.", r);
        return NULL;
    }
    const uint64_t p = row_find_geq(row, (uint64_t)r);
    if (p == row->count || row->e[p].col != (uint64_t)r)
    {
        PyErr_Format(PyExc_ValueError, "Row %zd has no diagonal entry.", r);
        return NULL;
    }
    /* Blocks right of the diagonal become D^{-1} B (src/block_system.c:1083-1130), all in one
     * batched device call. */
    const uint64_t m = bsize(s, r);
    int st = HYB_SUCCESS;
    const uint64_t nb = row->count - p - 1;
    if (nb > 0)
    {
        double **bs = (double **)PyMem_RawMalloc(nb * sizeof(double *));
        uint64_t *nc = (uint64_t *)PyMem_RawMalloc(nb * sizeof(uint64_t));
        if (!bs || !nc)
            st = HYB_FAILED_ALLOC;
        for (uint64_t j = 0; st == HYB_SUCCESS && j < nb; ++j)
        {
            bs[j] = row->e[p + 1 + j].vals;
            nc[j] = bsize(s, row->e[p + 1 + j].col);
        }
        if (st == HYB_SUCCESS)
        {
            Py_BEGIN_ALLOW_THREADS;
            st = hyb_block_lu_solve_batched(m, row->e[p].vals, nb, nc, bs, HYB_MEMORY_HOST);
            Py_END_ALLOW_THREADS;
        }
        PyMem_RawFree(bs);
        PyMem_RawFree(nc);
    }
    if (st)
        return raise_status(st, "row_apply_decomposition"), NULL;
    Py_RETURN_NONE;
}

/* ------------------------------------------------------------------------------- */
/* decomposition and solve                                                         */

static int parse_precision(PyObject *obj, int *out)
{
    if (!obj)
        return 0;
    if (!PyUnicode_Check(obj))
    {
        PyErr_SetString(PyExc_TypeError, "precision must be a string.");
        return -1;
    }
    const char *p = PyUnicode_AsUTF8(obj);
    if (!p)
        return -1;
    if (strcmp(p, "fp64") == 0)
        *out = HYB_PRECISION_FP64;
    else if (strcmp(p, "mixed") == 0)
        *out = HYB_PRECISION_MIXED;
    else
    {
        PyErr_Format(PyExc_ValueError, "Unknown precision '%s' (expected 'fp64' or 'mixed').", p);
        return -1;
    }
    return 0;
}

/* Uploads the host rows (pattern + values in CSR order) to a new device system. */
static int upload(bs_object *s, hyb_system **out)
{
    const uint64_t n = s->n;
    uint64_t nnz = 0, nval = 0;
    for (uint64_t i = 0; i < n; ++i)
    {
        nnz += s->rows[i].count;
        for (uint64_t j = 0; j < s->rows[i].count; ++j)
            nval += bsize(s, i) * bsize(s, s->rows[i].e[j].col);
    }
    uint64_t *sizes = (uint64_t *)PyMem_RawMalloc(n * sizeof(uint64_t));
    uint64_t *row_ptr = (uint64_t *)PyMem_RawMalloc((n + 1) * sizeof(uint64_t));
    uint64_t *cols = (uint64_t *)PyMem_RawMalloc((nnz + 1) * sizeof(uint64_t));
    double *vals = (double *)PyMem_RawMalloc((nval + 1) * sizeof(double));
    int st = HYB_FAILED_ALLOC;
    if (sizes && row_ptr && cols && vals)
    {
        uint64_t b = 0, v = 0;
        for (uint64_t i = 0; i < n; ++i)
        {
            sizes[i] = bsize(s, i);
            row_ptr[i] = b;
            for (uint64_t j = 0; j < s->rows[i].count; ++j, ++b)
            {
                const uint64_t cnt = bsize(s, i) * bsize(s, s->rows[i].e[j].col);
                cols[b] = s->rows[i].e[j].col;
                memcpy(vals + v, s->rows[i].e[j].vals, cnt * sizeof(double));
                v += cnt;
            }
        }
        row_ptr[n] = b;
        Py_BEGIN_ALLOW_THREADS;
        st = hyb_system_create(n, sizes, row_ptr, cols, out);
        if (st == HYB_SUCCESS)
        {
            st = hyb_system_set_values(*out, vals, HYB_MEMORY_HOST);
            if (st != HYB_SUCCESS)
            {
                hyb_system_destroy(*out);
                *out = NULL;
            }
        }
        Py_END_ALLOW_THREADS;
    }
    PyMem_RawFree(sizes);
    PyMem_RawFree(row_ptr);
    PyMem_RawFree(cols);
    PyMem_RawFree(vals);
    return st;
}

static PyObject *bs_decompose(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                              PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s || ensure_not_decomposed(s) < 0)
        return NULL;
    Py_ssize_t n_threads = 0;
    PyObject *prec_obj = NULL;
    const argspec_t spec[] = {{ARG_SSIZE, "n_threads", &n_threads, 1, 0}, {ARG_OBJECT, "precision", &prec_obj, 1, 1}, {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0)
        return NULL;
    if (n_threads < 0)
    {
        PyErr_SetString(PyExc_ValueError, "Number of threads must be non-negative.");
        return NULL;
    }
    int precision = HYB_PRECISION_FP64;
    if (parse_precision(prec_obj, &precision) < 0)
        return NULL;
    hyb_system *dev = NULL;
    int st = upload(s, &dev);
    if (st == HYB_SUCCESS)
    {
        Py_BEGIN_ALLOW_THREADS;
        st = hyb_decompose(dev, precision, &s->dinfo);
        if (st != HYB_SUCCESS)
        {
            hyb_system_destroy(dev);
            dev = NULL;
        }
        Py_END_ALLOW_THREADS;
    }
    if (st != HYB_SUCCESS)
    {
        if (st == HYB_CUDA_ERROR || st == HYB_NO_DEVICE)
            PyErr_Format(PyExc_RuntimeError, "Block system decomposition failed with error %d (%s: %s).", st,
                         hyb_status_string(st), hyb_last_cuda_error());
        else
            PyErr_Format(PyExc_RuntimeError, "Block system decomposition failed with error %d.", st);
        return NULL;
    }
    s->dev = dev;
    s->precision = precision;
    rows_free(s->rows, s->n);
    s->rows = NULL;
    Py_RETURN_NONE;
}

static PyObject *bs_operations(PyObject *self, PyTypeObject *cls, PyObject *const *Py_UNUSED(args), Py_ssize_t nargs,
                               PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s || ensure_decomposed(s) < 0 || no_args(nargs, kwnames, "No arguments accepted.") < 0)
        return NULL;
    uint64_t nops = 0;
    int st = hyb_operations(s->dev, &nops, NULL);
    if (st)
        return raise_status(st, "operations"), NULL;
    int64_t *ops = (int64_t *)PyMem_RawMalloc((2 * nops + 1) * sizeof(int64_t));
    if (!ops)
        return PyErr_NoMemory();
    st = hyb_operations(s->dev, &nops, ops);
    if (st)
    {
        PyMem_RawFree(ops);
        return raise_status(st, "operations"), NULL;
    }
    PyObject *t = PyTuple_New((Py_ssize_t)nops);
    for (uint64_t i = 0; t && i < nops; ++i)
    {
        PyObject *op = ops[2 * i + 1] < 0 ? Py_BuildValue("(n)", (Py_ssize_t)ops[2 * i])
                                          : Py_BuildValue("(nn)", (Py_ssize_t)ops[2 * i], (Py_ssize_t)ops[2 * i + 1]);
        if (!op)
        {
            Py_CLEAR(t);
            break;
        }
        PyTuple_SET_ITEM(t, (Py_ssize_t)i, op);
    }
    PyMem_RawFree(ops);
    return t;
}

static PyObject *bs_solve(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                          PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s || ensure_decomposed(s) < 0)
        return NULL;
    PyObject *val, *out_obj = NULL;
    double tol = 1e-12;
    Py_ssize_t max_iter = 50;
    const argspec_t spec[] = {{ARG_OBJECT, "val", &val, 0, 0},
                              {ARG_OBJECT, "out", &out_obj, 1, 0},
                              {ARG_DOUBLE, "tol", &tol, 1, 1},
                              {ARG_SSIZE, "max_iter", &max_iter, 1, 1},
                              {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0)
        return NULL;
    if (out_obj && !PyArray_Check(out_obj))
    {
        PyErr_SetString(PyExc_TypeError, "Argument 'out' must be of type numpy.ndarray.");
        return NULL;
    }
    if (max_iter < 0)
    {
        PyErr_SetString(PyExc_ValueError, "max_iter must be non-negative.");
        return NULL;
    }
    /* 1-D as in the reference (src/block_system.c:1288-1297); 2-D (dof, k) solves k
     * right-hand sides at once. */
    PyArrayObject *arr =
        (PyArrayObject *)PyArray_FROMANY(val, NPY_DOUBLE, 1, 2, NPY_ARRAY_ALIGNED | NPY_ARRAY_C_CONTIGUOUS);
    if (!arr)
        return NULL;
    const uint64_t dof = s->offsets[s->n];
    if ((uint64_t)PyArray_DIM(arr, 0) != dof || (PyArray_NDIM(arr) == 2 && PyArray_DIM(arr, 1) < 1))
    {
        PyErr_Format(PyExc_ValueError, "Array val must have %" PRIu64 " rows.", dof);
        Py_DECREF(arr);
        return NULL;
    }
    PyArrayObject *out = (PyArrayObject *)out_obj;
    if (out)
    {
        if (check_out(out, PyArray_NDIM(arr), PyArray_DIMS(arr), "out") < 0)
        {
            Py_DECREF(arr);
            return NULL;
        }
        Py_INCREF(out);
    }
    else
    {
        out = (PyArrayObject *)PyArray_SimpleNew(PyArray_NDIM(arr), PyArray_DIMS(arr), NPY_DOUBLE);
        if (!out)
        {
            Py_DECREF(arr);
            return NULL;
        }
    }
    const uint64_t nrhs = PyArray_NDIM(arr) == 2 ? (uint64_t)PyArray_DIM(arr, 1) : 1;
    int st;
    hyb_solve_info info = {0, -1.0, 0};
    Py_BEGIN_ALLOW_THREADS;
    st = hyb_solve(s->dev, (const double *)PyArray_DATA(arr), (double *)PyArray_DATA(out), nrhs, HYB_MEMORY_HOST, tol,
                   (uint32_t)max_iter, s->precision == HYB_PRECISION_MIXED ? &info : NULL);
    Py_END_ALLOW_THREADS;
    Py_DECREF(arr);
    s->sinfo = info;
    s->solve_status = st;
    if (st != HYB_SUCCESS)
    {
        if (st == HYB_NOT_CONVERGED)
            PyErr_Format(PyExc_RuntimeError,
                         "Iterative refinement did not reach the tolerance %g in %u steps (relative residual %g).",
                         tol, info.iterations, info.relative_residual);
        else
            raise_status(st, "solve");
        Py_DECREF(out);
        return NULL;
    }
    return (PyObject *)out;
}

static PyObject *bs_copy(PyObject *self, PyTypeObject *cls, PyObject *const *Py_UNUSED(args), Py_ssize_t nargs,
                         PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s || no_args(nargs, kwnames, "No arguments accepted.") < 0)
        return NULL;
    PyTypeObject *tp = Py_TYPE(self);
    bs_object *t = (bs_object *)tp->tp_alloc(tp, 0);
    if (!t)
        return NULL;
    t->n = s->n;
    t->precision = s->precision;
    t->dinfo = s->dinfo;
    t->offsets = (uint64_t *)PyMem_Malloc((s->n + 1) * sizeof(uint64_t));
    if (!t->offsets)
    {
        Py_DECREF(t);
        return PyErr_NoMemory();
    }
    memcpy(t->offsets, s->offsets, (s->n + 1) * sizeof(uint64_t));
    if (s->dev)
    {
        int st;
        Py_BEGIN_ALLOW_THREADS;
        st = hyb_system_copy(s->dev, &t->dev);
        Py_END_ALLOW_THREADS;
        if (st)
        {
            Py_DECREF(t);
            return raise_status(st, "copy"), NULL;
        }
        return (PyObject *)t;
    }
    t->rows = (hrow_t *)PyMem_RawCalloc(s->n, sizeof(hrow_t));
    if (!t->rows)
    {
        Py_DECREF(t);
        return PyErr_NoMemory();
    }
    for (uint64_t i = 0; i < s->n; ++i)
    {
        const hrow_t *src = s->rows + i;
        hrow_t *dst = t->rows + i;
        if (row_reserve(dst, src->count) < 0)
        {
            Py_DECREF(t);
            return PyErr_NoMemory();
        }
        for (uint64_t j = 0; j < src->count; ++j)
        {
            const uint64_t cnt = bsize(s, i) * bsize(s, src->e[j].col);
            double *v = (double *)PyMem_RawMalloc(cnt * sizeof(double) + 8);
            if (!v)
            {
                Py_DECREF(t);
                return PyErr_NoMemory();
            }
            memcpy(v, src->e[j].vals, cnt * sizeof(double));
            dst->e[j].col = src->e[j].col;
            dst->e[j].vals = v;
            dst->count += 1;
        }
    }
    return (PyObject *)t;
}

/* ------------------------------------------------------------------------------- */
/* ordering                                                                        */

static int cmp_entry(const void *a, const void *b)
{
    const uint64_t x = ((const entry_t *)a)->col, y = ((const entry_t *)b)->col;
    return x < y ? -1 : (x > y);
}

static PyArrayObject *as_order(const bs_object *s, PyObject *obj)
{
    PyArrayObject *arr =
        (PyArrayObject *)PyArray_FROMANY(obj, NPY_UINT64, 1, 1, NPY_ARRAY_ALIGNED | NPY_ARRAY_C_CONTIGUOUS);
    if (!arr)
        return NULL;
    if ((uint64_t)PyArray_DIM(arr, 0) != s->n)
    {
        PyErr_Format(PyExc_ValueError, "Array new_order must have %" PRIu64 " entries.", s->n);
        Py_DECREF(arr);
        return NULL;
    }
    return arr;
}

static PyObject *bs_reorder_blocks(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                                   PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s || ensure_not_decomposed(s) < 0)
        return NULL;
    PyObject *order_obj;
    Py_ssize_t n_threads = 0;
    const argspec_t spec[] = {{ARG_OBJECT, "new_order", &order_obj, 0, 0}, {ARG_SSIZE, "n_threads", &n_threads, 1, 0}, {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0)
        return NULL;
    if (n_threads < 0)
    {
        PyErr_SetString(PyExc_ValueError, "Number of threads must be non-negative.");
        return NULL;
    }
    PyArrayObject *arr = as_order(s, order_obj);
    if (!arr)
        return NULL;
    const uint64_t *order = (const uint64_t *)PyArray_DATA(arr);
    const uint64_t n = s->n;
    unsigned char *seen = (unsigned char *)PyMem_RawCalloc(n, 1);
    hrow_t *rows = (hrow_t *)PyMem_RawMalloc(n * sizeof(hrow_t));
    uint64_t *sizes = (uint64_t *)PyMem_RawMalloc(n * sizeof(uint64_t));
    if (!seen || !rows || !sizes)
    {
        PyMem_RawFree(seen);
        PyMem_RawFree(rows);
        PyMem_RawFree(sizes);
        Py_DECREF(arr);
        return PyErr_NoMemory();
    }
    /* Duplicate check of src/block_system.c:1498-1517; indices out of range are rejected
     * too (the reference does not check them). */
    for (uint64_t i = 0; i < n; ++i)
    {
        if (order[i] >= n || seen[order[i]])
        {
            if (order[i] >= n)
                PyErr_Format(PyExc_ValueError, "Order index %" PRIu64 " is out of range.", order[i]);
            else
                PyErr_Format(PyExc_ValueError, "Duplicate order index %" PRIu64 ".", order[i]);
            PyMem_RawFree(seen);
            PyMem_RawFree(rows);
            PyMem_RawFree(sizes);
            Py_DECREF(arr);
            return NULL;
        }
        seen[order[i]] = 1;
    }
    /* Renumber columns, sort each row, move row i to order[i] (src/block_system.c:1522-1637). */
    Py_BEGIN_ALLOW_THREADS;
    for (uint64_t i = 0; i < n; ++i)
    {
        hrow_t *r = s->rows + i;
        for (uint64_t j = 0; j < r->count; ++j)
            r->e[j].col = order[r->e[j].col];
        qsort(r->e, r->count, sizeof(entry_t), cmp_entry);
        rows[order[i]] = *r;
        sizes[order[i]] = bsize(s, i);
    }
    memcpy(s->rows, rows, n * sizeof(hrow_t));
    for (uint64_t i = 0; i < n; ++i)
        s->offsets[i + 1] = s->offsets[i] + sizes[i];
    Py_END_ALLOW_THREADS;
    PyMem_RawFree(seen);
    PyMem_RawFree(rows);
    PyMem_RawFree(sizes);
    Py_DECREF(arr);
    Py_RETURN_NONE;
}

static PyObject *bs_compute_reordering(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                                       PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s || ensure_not_decomposed(s) < 0)
        return NULL;
    PyObject *strat_obj = NULL;
    Py_ssize_t max_colors = 0;
    const argspec_t spec[] = {
        {ARG_OBJECT, "strategy", &strat_obj, 1, 0}, {ARG_SSIZE, "max_colors", &max_colors, 1, 0}, {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0)
        return NULL;
    int strategy = HYB_ORDERING_FIRST;
    if (strat_obj)
    {
        if (!PyUnicode_Check(strat_obj))
        {
            PyErr_SetString(PyExc_TypeError, "Ordering strategy must be a string.");
            return NULL;
        }
        const char *name = PyUnicode_AsUTF8(strat_obj);
        if (!name)
            return NULL;
        if (strcmp(name, "greedy") == 0)
            strategy = HYB_ORDERING_GREEDY;
        else if (strcmp(name, "balanced") == 0)
            strategy = HYB_ORDERING_BALANCED;
        else if (strcmp(name, "first") == 0)
            strategy = HYB_ORDERING_FIRST;
        else
        {
            PyErr_Format(PyExc_ValueError, "Unknown ordering strategy '%s'.", name);
            return NULL;
        }
    }
    if (max_colors < 0)
    {
        PyErr_SetString(PyExc_ValueError, "Maximum number of colors must be non-negative.");
        return NULL;
    }
    const uint64_t n = s->n;
    uint64_t nnz = 0;
    for (uint64_t i = 0; i < n; ++i)
        nnz += s->rows[i].count;
    /* 0 means "as many colors as the longest row" (src/block_system.c:1725-1733). */
    if (max_colors == 0)
        for (uint64_t i = 0; i < n; ++i)
            max_colors = (Py_ssize_t)s->rows[i].count > max_colors ? (Py_ssize_t)s->rows[i].count : max_colors;
    uint64_t *row_ptr = (uint64_t *)PyMem_RawMalloc((n + 1) * sizeof(uint64_t));
    uint64_t *cols = (uint64_t *)PyMem_RawMalloc((nnz + 1) * sizeof(uint64_t));
    const npy_intp dim = (npy_intp)n;
    PyArrayObject *arr = (PyArrayObject *)PyArray_SimpleNew(1, &dim, NPY_UINT64);
    if (!row_ptr || !cols || !arr)
    {
        PyMem_RawFree(row_ptr);
        PyMem_RawFree(cols);
        Py_XDECREF(arr);
        return PyErr_NoMemory();
    }
    uint64_t b = 0;
    for (uint64_t i = 0; i < n; ++i)
    {
        row_ptr[i] = b;
        for (uint64_t j = 0; j < s->rows[i].count; ++j)
            cols[b++] = s->rows[i].e[j].col;
    }
    row_ptr[n] = b;
    int st;
    if (max_colors == 0)
        st = HYB_MAX_COLORS;
    else
        st = hyb_compute_ordering(n, row_ptr, cols, strategy, (uint64_t)max_colors, (uint64_t *)PyArray_DATA(arr));
    PyMem_RawFree(row_ptr);
    PyMem_RawFree(cols);
    if (st != HYB_SUCCESS)
    {
        Py_DECREF(arr);
        if (st == HYB_MAX_COLORS)
            PyErr_Format(PyExc_ValueError, "Maximum number of colors (%zd) exceeded.", max_colors);
        else
            PyErr_SetString(PyExc_RuntimeError, "Unknown error occurred.");
        return NULL;
    }
    return (PyObject *)arr;
}

/* Shared argument handling of reorder_vector / unorder_vector (src/block_system.c:1822-1908). */
static int prepare_vector(bs_object *s, PyObject *const *args, Py_ssize_t nargs, PyObject *kwnames,
                          PyArrayObject **p_order, PyArrayObject **p_vec, PyArrayObject **p_out)
{
    PyObject *order_obj, *vec_obj, *out_obj = NULL;
    const argspec_t spec[] = {{ARG_OBJECT, "new_order", &order_obj, 0, 0},
                              {ARG_OBJECT, "vector", &vec_obj, 0, 0},
                              {ARG_OBJECT, "out", &out_obj, 1, 0},
                              {0}};
    if (parse_args(args, nargs, kwnames, spec) < 0)
        return -1;
    if (out_obj && !PyArray_Check(out_obj))
    {
        PyErr_SetString(PyExc_TypeError, "Argument 'out' must be of type numpy.ndarray.");
        return -1;
    }
    PyArrayObject *order = as_order(s, order_obj);
    if (!order)
        return -1;
    const uint64_t *o = (const uint64_t *)PyArray_DATA(order);
    for (uint64_t i = 0; i < s->n; ++i)
        if (o[i] >= s->n)
        {
            PyErr_Format(PyExc_ValueError, "Order index %" PRIu64 " is out of range.", o[i]);
            Py_DECREF(order);
            return -1;
        }
    const npy_intp dof = (npy_intp)s->offsets[s->n];
    PyArrayObject *vec =
        (PyArrayObject *)PyArray_FROMANY(vec_obj, NPY_DOUBLE, 1, 1, NPY_ARRAY_C_CONTIGUOUS | NPY_ARRAY_ALIGNED);
    if (!vec)
    {
        Py_DECREF(order);
        return -1;
    }
    if (PyArray_DIM(vec, 0) != dof)
    {
        PyErr_Format(PyExc_ValueError, "Array vector must have %zd entries.", (Py_ssize_t)dof);
        Py_DECREF(order);
        Py_DECREF(vec);
        return -1;
    }
    PyArrayObject *out = (PyArrayObject *)out_obj;
    if (out)
    {
        if (check_out(out, 1, &dof, "out") < 0)
        {
            Py_DECREF(order);
            Py_DECREF(vec);
            return -1;
        }
        Py_INCREF(out);
    }
    else if (!(out = (PyArrayObject *)PyArray_SimpleNew(1, &dof, NPY_DOUBLE)))
    {
        Py_DECREF(order);
        Py_DECREF(vec);
        return -1;
    }
    *p_order = order;
    *p_vec = vec;
    *p_out = out;
    return 0;
}

/* reorder_vector (src/block_system.c:1910-1941): the output walks blocks i = 0.. in the old
 * numbering and takes the segment the system now stores at order[i]: new layout -> old. */
static PyObject *bs_reorder_vector(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                                   PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    PyArrayObject *order, *vec, *out;
    if (!s || prepare_vector(s, args, nargs, kwnames, &order, &vec, &out) < 0)
        return NULL;
    const uint64_t *o = (const uint64_t *)PyArray_DATA(order);
    const double *v = (const double *)PyArray_DATA(vec);
    double *r = (double *)PyArray_DATA(out);
    uint64_t off = 0;
    for (uint64_t i = 0; i < s->n; ++i)
    {
        const uint64_t sz = bsize(s, o[i]);
        memmove(r + off, v + s->offsets[o[i]], sz * sizeof(double));
        off += sz;
    }
    Py_DECREF(order);
    Py_DECREF(vec);
    return (PyObject *)out;
}

/* unorder_vector (src/block_system.c:1966-1997): the inverse map, old layout -> new. */
static PyObject *bs_unorder_vector(PyObject *self, PyTypeObject *cls, PyObject *const *args, Py_ssize_t nargs,
                                   PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    PyArrayObject *order, *vec, *out;
    if (!s || prepare_vector(s, args, nargs, kwnames, &order, &vec, &out) < 0)
        return NULL;
    const uint64_t *o = (const uint64_t *)PyArray_DATA(order);
    const double *v = (const double *)PyArray_DATA(vec);
    double *r = (double *)PyArray_DATA(out);
    uint64_t off = 0;
    for (uint64_t i = 0; i < s->n; ++i)
    {
        const uint64_t sz = bsize(s, o[i]);
        memmove(r + s->offsets[o[i]], v + off, sz * sizeof(double));
        off += sz;
    }
    Py_DECREF(order);
    Py_DECREF(vec);
    return (PyObject *)out;
}

/* ------------------------------------------------------------------------------- */
/* extension-only introspection                                                    */

static PyObject *bs_last_decompose_info(PyObject *self, PyTypeObject *cls, PyObject *const *Py_UNUSED(args),
                                        Py_ssize_t nargs, PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s || ensure_decomposed(s) < 0 || no_args(nargs, kwnames, "No arguments accepted.") < 0)
        return NULL;
    const hyb_decompose_info *d = &s->dinfo;
    return Py_BuildValue("{s:s,s:K,s:K,s:K,s:d,s:K,s:K,s:L}", "precision",
                         s->precision == HYB_PRECISION_MIXED ? "mixed" : "fp64", "n_levels",
                         (unsigned long long)d->n_levels, "filled_blocks", (unsigned long long)d->filled_blocks,
                         "factor_values", (unsigned long long)d->factor_values, "factor_flops", d->factor_flops,
                         "zero_pivots", (unsigned long long)d->zero_pivots, "non_finite",
                         (unsigned long long)d->non_finite, "first_bad_pivot", (long long)d->first_bad_pivot);
}

static PyObject *bs_last_solve_info(PyObject *self, PyTypeObject *cls, PyObject *const *Py_UNUSED(args),
                                    Py_ssize_t nargs, PyObject *kwnames)
{
    bs_object *s = check_self(self, cls);
    if (!s || ensure_decomposed(s) < 0 || no_args(nargs, kwnames, "No arguments accepted.") < 0)
        return NULL;
    return Py_BuildValue("{s:I,s:d,s:O}", "iterations", s->sinfo.iterations, "relative_residual",
                         s->sinfo.relative_residual, "converged", s->solve_status == HYB_SUCCESS ? Py_True : Py_False);
}

static PyObject *bs_get_n_blocks(PyObject *self, void *Py_UNUSED(c))
{
    return PyLong_FromUnsignedLongLong(((bs_object *)self)->n);
}

static PyObject *bs_get_block_sizes(PyObject *self, void *Py_UNUSED(c))
{
    const bs_object *s = (bs_object *)self;
    const npy_intp dim = (npy_intp)s->n;
    PyArrayObject *arr = (PyArrayObject *)PyArray_SimpleNew(1, &dim, NPY_UINT64);
    if (!arr)
        return NULL;
    uint64_t *out = (uint64_t *)PyArray_DATA(arr);
    for (uint64_t i = 0; i < s->n; ++i)
        out[i] = bsize(s, i);
    return (PyObject *)arr;
}

static PyObject *bs_get_precision(PyObject *self, void *Py_UNUSED(c))
{
    const bs_object *s = (bs_object *)self;
    if (!s->dev)
        Py_RETURN_NONE;
    return PyUnicode_FromString(s->precision == HYB_PRECISION_MIXED ? "mixed" : "fp64");
}

#define METH(name, fn, doc) {name, (PyCFunction)(void (*)(void))fn, METH_METHOD | METH_FASTCALL | METH_KEYWORDS, doc}

static PyMethodDef bs_methods[] = {
    METH("add_block", bs_add_block,
         "add_block(row: int, col: int, val: numpy.typing.ArrayLike)\nAdd a block to the system (summed into an "
         "existing block)."),
    METH("add_blocks", bs_add_blocks,
         "add_blocks(rows: numpy.typing.ArrayLike, cols: numpy.typing.ArrayLike, values: numpy.typing.ArrayLike)\n"
         "Add many blocks: block i is (rows[i], cols[i]) with its row-major values next in the 1-D values "
         "(summed into existing blocks, in order). Not in the reference: a bulk form of add_block."),
    METH("is_valid", bs_is_valid, "is_valid() -> bool\nCheck if the system has symmetric sparsity and has diagonal blocks."),
    METH("as_array", bs_as_array, "as_array() -> numpy.typing.NDArray[numpy.double]\nReturn the system as a full matrix."),
    METH("get_row_block_indices", bs_get_row_block_indices,
         "get_row_block_indices(row: int) -> tuple[int, ...]\nColumn block indices of the row."),
    METH("get_block", bs_get_block, "get_block(row: int, col: int) -> numpy.typing.NDArray[numpy.double]\nCopy of a block."),
    METH("get_block_size", bs_get_block_size, "get_block_size(row: int, col: int) -> tuple[int, int]\nSize of a block."),
    METH("multiply_row", bs_multiply_row,
         "multiply_row(row: int, val: numpy.typing.ArrayLike, start: int = 0) -> None\nLeft-multiply the row's blocks "
         "at or after column `start` by a square matrix."),
    METH("eliminate_row", bs_eliminate_row,
         "eliminate_row(row_src: int, row_tgt: int, val: numpy.typing.ArrayLike) -> None\nM_t <- M_t - val @ M_s over "
         "the columns after row_src, creating fill."),
    METH("has_block", bs_has_block, "has_block(row: int, col: int) -> bool\nWhether block (row, col) is present."),
    METH("no_lower_connections", bs_no_lower_connections,
         "no_lower_connections() -> numpy.typing.NDArray[numpy.bool]\nRows without blocks left of the diagonal."),
    METH("first_column", bs_first_column, "first_column(row: int) -> int\nFirst column index of a non-empty row."),
    METH("get_next_column_index", bs_get_next_column_index,
         "get_next_column_index(row: int, col: int) -> int\nColumn index after `col` in the row."),
    METH("decompose_diagonal", bs_decompose_diagonal,
         "decompose_diagonal(idx: int) -> None\nUnpivoted LU of the diagonal block (on the GPU)."),
    METH("solve_diagonal", bs_solve_diagonal,
         "solve_diagonal(idx: int, val, out=None) -> numpy.typing.NDArray[numpy.double]\nSolve with the factored "
         "diagonal block; returns the output array (the reference returns None)."),
    METH("row_apply_decomposition", bs_row_apply_decomposition,
         "row_apply_decomposition(row: int) -> None\nApply the factored diagonal to the blocks right of it."),
    METH("decompose", bs_decompose,
         "decompose(n_threads: int = 0, *, precision: str = 'fp64') -> None\nFactor the block system on the GPU. "
         "n_threads is accepted for compatibility; precision 'mixed' factors in FP32 and refines in FP64."),
    METH("operations", bs_operations,
         "operations() -> tuple[tuple[int, int] | tuple[int], ...]\nThe elimination operations in the reference's "
         "single-thread order."),
    METH("solve", bs_solve,
         "solve(val, out=None, *, tol: float = 1e-12, max_iter: int = 50) -> numpy.typing.NDArray[numpy.double]\n"
         "Solve with the decomposition. val may be 1-D (dof,) or 2-D (dof, k); tol and max_iter drive the mixed "
         "form's refinement."),
    METH("copy", bs_copy, "copy() -> BlockSystem\nCreate a copy of the system."),
    METH("reorder_blocks", bs_reorder_blocks,
         "reorder_blocks(new_order: numpy.typing.ArrayLike, n_threads: int = 0)\nRenumber blocks: old i becomes "
         "new_order[i]."),
    METH("compute_reordering", bs_compute_reordering,
         "compute_reordering(strategy='first', max_colors: int = 0) -> numpy.typing.NDArray[numpy.uint64]\nColoring "
         "order of the blocks (bit-exact with the reference)."),
    METH("reorder_vector", bs_reorder_vector,
         "reorder_vector(new_order, vector, out=None)\nMap a vector from the current block layout back to the layout "
         "before reorder_blocks(new_order)."),
    METH("unorder_vector", bs_unorder_vector,
         "unorder_vector(new_order, vector, out=None)\nMap a vector from the layout before reorder_blocks(new_order) "
         "to the current one."),
    METH("last_decompose_info", bs_last_decompose_info, "last_decompose_info() -> dict\nSchedule and pivot statistics."),
    METH("last_solve_info", bs_last_solve_info,
         "last_solve_info() -> dict\nRefinement iterations and FP64 relative residual of the last mixed solve."),
    {NULL, NULL, 0, NULL},
};

static PyGetSetDef bs_getset[] = {
    {"n_blocks", bs_get_n_blocks, NULL, "int : Number of blocks.", NULL},
    {"block_sizes", bs_get_block_sizes, NULL, "numpy.typing.NDArray[numpy.uint64] : Array of sizes of blocks.", NULL},
    {"precision", bs_get_precision, NULL, "str | None : Precision of the decomposition, None before decompose().",
     NULL},
    {NULL, NULL, NULL, NULL, NULL},
};

static PyType_Slot bs_slots[] = {
    {Py_tp_new, bs_new},
    {Py_tp_dealloc, bs_dealloc},
    {Py_tp_traverse, pymod_traverse_type},
    {Py_tp_methods, bs_methods},
    {Py_tp_getset, bs_getset},
    {Py_tp_doc, "BlockSystem(*block_sizes: int)\nBlock system for hybridized solver (factored on a B200)."},
    {0, NULL},
};

PyType_Spec pymod_block_system_spec = {
    .name = "hybsol._mod.BlockSystem",
    .basicsize = sizeof(bs_object),
    .itemsize = 0,
    .flags = Py_TPFLAGS_HEAPTYPE | Py_TPFLAGS_HAVE_GC | Py_TPFLAGS_IMMUTABLETYPE | Py_TPFLAGS_DEFAULT,
    .slots = bs_slots,
};
