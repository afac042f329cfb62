// Stand-in for Intel MKL's umbrella header, used only to compile the
// reference's own sources into the oracle library (oracle/_ref).  The
// reference includes <mkl.h> but calls no MKL routine on the IVF path
// (its cblas_sdot call is commented out in utils.h); it relies on the
// standard headers MKL happens to pull in, so this header provides those.
#pragma once
#include <functional>
#include <iomanip>
#include <sstream>
#include <omp.h>
#include <climits>
#include <queue>
#include <unistd.h>
