// Error text of host-only entry points (no context): read back by rls_last_error(NULL).
#pragma once
#include <string>

void rls_host_error(const std::string& msg);
