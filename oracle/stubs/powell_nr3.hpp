// ORACLE / TEST INFRASTRUCTURE ONLY.
// Stand-in for toofus' powell_nr3.hpp (included at src/p-tracker.hpp:51 of the
// reference; toofus is not vendored and has no pinned version).  Exposes the
// project-written Powell minimiser under the name the reference uses.
#pragma once
#include "../powell.hpp"
using ptk_oracle::Powell;
