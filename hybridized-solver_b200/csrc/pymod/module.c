/*
 * module.c - multi-phase initialisation of `hybsol._mod` (the reference's module entry,
 * src/module.c:25-63): module state holding the two heap types, several interpreters allowed.
 */
#define HYBSOL_IMPORT_ARRAY
#include "pymod.h"

static int module_exec(PyObject *mod)
{
    if (PyArray_ImportNumPyAPI() < 0)
        return -1;
    pymod_state *st = (pymod_state *)PyModule_GetState(mod);
    if (!st)
        return -1;
    PyTypeObject *info = (PyTypeObject *)PyType_FromModuleAndSpec(mod, &pymod_block_info_spec, NULL);
    if (!info || PyModule_AddType(mod, info) < 0)
    {
        Py_XDECREF(info);
        return -1;
    }
    st->type_block_info = info;
    PyTypeObject *sys = (PyTypeObject *)PyType_FromModuleAndSpec(mod, &pymod_block_system_spec, NULL);
    if (!sys || PyModule_AddType(mod, sys) < 0)
    {
        Py_XDECREF(sys);
        return -1;
    }
    st->type_block_system = sys;
    if (PyModule_AddIntConstant(mod, "ABI_VERSION", hyb_version()) < 0)
        return -1;
    return 0;
}

static int module_traverse(PyObject *mod, visitproc visit, void *arg)
{
    pymod_state *st = (pymod_state *)PyModule_GetState(mod);
    if (st)
    {
        Py_VISIT(st->type_block_info);
        Py_VISIT(st->type_block_system);
    }
    return 0;
}

static int module_clear(PyObject *mod)
{
    pymod_state *st = (pymod_state *)PyModule_GetState(mod);
    if (st)
    {
        Py_CLEAR(st->type_block_info);
        Py_CLEAR(st->type_block_system);
    }
    return 0;
}

static void module_free(void *mod)
{
    module_clear((PyObject *)mod);
}

static PyObject *mod_device_available(PyObject *Py_UNUSED(self), PyObject *Py_UNUSED(args))
{
    return PyBool_FromLong(hyb_device_available());
}

static PyMethodDef module_methods[] = {
    {"device_available", mod_device_available, METH_NOARGS, "device_available() -> bool\nWhether an sm_100 GPU is visible."},
    {NULL, NULL, 0, NULL},
};

static PyModuleDef_Slot module_slots[] = {
    {Py_mod_exec, module_exec},
    {Py_mod_multiple_interpreters, Py_MOD_MULTIPLE_INTERPRETERS_SUPPORTED},
    {0, NULL},
};

PyModuleDef pymod_def = {
    PyModuleDef_HEAD_INIT,
    .m_name = "hybsol._mod",
    .m_doc = "B200 block-sparse LU for the hybridized solver (drop-in for the reference extension).",
    .m_size = sizeof(pymod_state),
    .m_methods = module_methods,
    .m_slots = module_slots,
    .m_traverse = module_traverse,
    .m_clear = module_clear,
    .m_free = module_free,
};

int pymod_traverse_type(PyObject *self, visitproc visit, void *arg)
{
    Py_VISIT(Py_TYPE(self));
    return 0;
}

PyMODINIT_FUNC PyInit__mod(void)
{
    return PyModuleDef_Init(&pymod_def);
}
