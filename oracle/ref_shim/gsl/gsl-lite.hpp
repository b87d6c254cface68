// The same stand-in under the include path some reference headers use (see ../gsl-lite/gsl-lite.hpp).
#pragma once
#include "../gsl-lite/gsl-lite.hpp"
