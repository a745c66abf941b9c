// Stand-in for the reference's include/FSI_Simulator/utils/Logger.hpp when
// its fluid-step sources are compiled into oracle/_ref: the reference logs
// through spdlog (not installed here); these macros discard the messages.
// ASSERT is a no-op, as in the reference's release builds.
#pragma once

#define LOG_TRACE(...) ((void)0)
#define LOG_DEBUG(...) ((void)0)
#define LOG_INFO(...) ((void)0)
#define LOG_WARN(...) ((void)0)
#define LOG_ERROR(...) ((void)0)
#define LOG_CRITICAL(...) ((void)0)
#define ASSERT(condition, ...) ((void)0)
