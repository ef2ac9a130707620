// Sets the text mass_lb_last_error() returns on the calling thread (api.cu).
#pragma once
#include <string>
void mlb_set_last_error(const std::string& msg);
