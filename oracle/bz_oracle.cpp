// ORACLE — test infrastructure only. Bezier restatement (filled in below).
#include "bz_oracle.hpp"
