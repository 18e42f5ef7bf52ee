// Fortran list-directed output of REAL(8) values as the reference's gfortran
// build writes them (`write(unit,*) a, b, ...`): every item is one blank and
// a 25-character G field with 17 significant digits (F form with five
// trailing blanks for 0.1 <= |x| < 1e17, else d.dddE+ddd).
#pragma once
#include <string>

namespace tara {
// appends the items of one record (no newline)
void list_directed_append(std::string& out, const double* v, int n);
}  // namespace tara
