// The library's last-error message (dsx_last_error), for the parts of the
// library built outside dsx_engine.cu.
#pragma once

namespace dsx {
void set_last_error(const char* message);
}
