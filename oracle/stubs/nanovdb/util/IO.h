// Test-infrastructure shim (oracle build only); see ../NanoVDB.h.
#pragma once
#include "../NanoVDB.h"
