/*
 * pymod.h - the `hybsol._mod` CPython extension: the reference's Python surface
 * (`hybsol._mod.BlockSystem`, `hybsol._mod.BlockInfo`; src/module.c, src/block_system.c,
 * src/block_info.c, typed in python/hybsol/_mod.pyi) over the C ABI of hybsol_b200.h.
 *
 * Host memory holds the block rows while a system is assembled (add_block, reordering,
 * the fine-grained row operations). decompose() hands the pattern and values to the
 * device library; from then on the factors live on the GPU and accessors read them back.
 */
#pragma once

#ifndef PY_SSIZE_T_CLEAN
#define PY_SSIZE_T_CLEAN
#endif
#define NPY_NO_DEPRECATED_API NPY_1_7_API_VERSION
#ifndef HYBSOL_IMPORT_ARRAY
#define NO_IMPORT_ARRAY
#endif
#define PY_ARRAY_UNIQUE_SYMBOL hybsol_b200_ARRAY_API

#include <Python.h>
#include <numpy/arrayobject.h>
#include <stdint.h>

#include "hybsol_b200.h"

#define PYMOD_INTERNAL __attribute__((visibility("hidden")))

typedef struct
{
    PyTypeObject *type_block_info;
    PyTypeObject *type_block_system;
} pymod_state;

PYMOD_INTERNAL extern PyModuleDef pymod_def;
PYMOD_INTERNAL extern PyType_Spec pymod_block_system_spec;
PYMOD_INTERNAL extern PyType_Spec pymod_block_info_spec;
PYMOD_INTERNAL int pymod_traverse_type(PyObject *self, visitproc visit, void *arg);

static inline const pymod_state *pymod_state_of(PyTypeObject *type)
{
    PyObject *mod = PyType_GetModuleByDef(type, &pymod_def);
    return mod ? (const pymod_state *)PyModule_GetState(mod) : NULL;
}
