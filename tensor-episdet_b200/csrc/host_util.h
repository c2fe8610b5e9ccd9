// host_util.h -- error reporting shared by the host-side sources.
#pragma once
#include <cstdarg>
#include <cstdio>

#include "episdet.h"

namespace episdet {

// Records a thread-local message for episdet_last_error() and returns `s`.
episdet_status set_error(episdet_status s, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
void clear_error();

}  // namespace episdet
