// Stand-in (no content needed by the guided-path functions under test).
#pragma once
#include "../common.h"
