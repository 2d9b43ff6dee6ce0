// Oracle (test infrastructure only): the linear-solver context surface the
// reference's assembler.h includes (from the absent liblinsolve submodule),
// provided by this library's reconstruction of it.
#pragma once
#include "compat/linearSolverContext.h"
