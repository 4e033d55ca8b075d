// Stand-in for <Python.h> (test infrastructure only): nothing of it is used
// by the grid kernels the harness compiles.
#pragma once
