/* Test-only module init for the reference's own C implementation of the grid
 * hot path.  This file is project-written; it is the only source under oracle/
 * that is linked together with the reference's files
 *   c/bmgs/bmgs.c  c/bc.c  c/operators.c  c/transformers.c  c/woperators.c
 * which are compiled in place (never copied) by oracle/Makefile.
 *
 * It registers exactly the three constructors that the reference's module
 * table registers for this path (c/_gpaw.c:154 "Operator", :155 "WOperator",
 * :157 "Transformer") under the module name `_gpaw_ref`, so the reference's
 * Python call sites (gpaw/fd_operators.py:75-77, gpaw/transformers.py:71-76,
 * gpaw/wfd_operators.py:70-74) can be restated against it unchanged.
 *
 * This is the oracle: test infrastructure, imported only by tests/, the smoke
 * check and the CPU-baseline leg of bench.py.
 */
#include <Python.h>
#define PY_ARRAY_UNIQUE_SYMBOL GPAW_ARRAY_API
#include <numpy/arrayobject.h>

extern PyTypeObject OperatorType;
extern PyTypeObject WOperatorType;
extern PyTypeObject TransformerType;
PyObject *NewOperatorObject(PyObject *obj, PyObject *args);
PyObject *NewWOperatorObject(PyObject *obj, PyObject *args);
PyObject *NewTransformerObject(PyObject *obj, PyObject *args);

static PyMethodDef ref_functions[] = {
    {"Operator", NewOperatorObject, METH_VARARGS, 0},
    {"WOperator", NewWOperatorObject, METH_VARARGS, 0},
    {"Transformer", NewTransformerObject, METH_VARARGS, 0},
    {NULL, NULL, 0, NULL}};

static struct PyModuleDef ref_module = {
    PyModuleDef_HEAD_INIT, "_gpaw_ref",
    "Reference GPAW grid operators (oracle only)", -1, ref_functions};

PyMODINIT_FUNC PyInit__gpaw_ref(void)
{
    import_array();
    if (PyType_Ready(&OperatorType) < 0)
        return NULL;
    if (PyType_Ready(&WOperatorType) < 0)
        return NULL;
    if (PyType_Ready(&TransformerType) < 0)
        return NULL;
    return PyModule_Create(&ref_module);
}
