// Error reporting shared by the library's translation units: records the
// message that ifdtd_last_error returns on the calling thread, returns code.
#pragma once

#include <string>

namespace ifdtd {
int record_error(int code, const std::string& msg);
}
