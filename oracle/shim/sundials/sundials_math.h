#include "../sundials_shim.h"
