// ORACLE — test infrastructure only (see oracle.hpp). Bezier smoother restatement.
#pragma once
namespace orc {}
