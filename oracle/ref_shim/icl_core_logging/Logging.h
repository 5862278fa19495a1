// No-op logging macros in place of icl_core_logging (oracle/_ref build only).
#pragma once
#include <cstdint>
#include "ThreadStream.h"
#define DECLARE_LOG_STREAM(x)
#define LOGGING_ERROR(...)
#define LOGGING_WARNING(...)
#define LOGGING_INFO(...)
#define LOGGING_DEBUG(...)
#define LOGGING_TRACE(...)
#define LOGGING_ERROR_C(...)
#define LOGGING_WARNING_C(...)
#define LOGGING_INFO_C(...)
#define LOGGING_DEBUG_C(...)
#define LOGGING_TRACE_C(...)
