// ORACLE BUILD SHIM (test infrastructure): see root_stub.h.
#pragma once
#include "root_stub.h"
