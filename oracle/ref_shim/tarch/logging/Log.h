// Logging stand-in for tarch::logging::Log: warnings and errors go to stderr.
// Test infrastructure for oracle/_ref only.
#pragma once
#include <iostream>
#include <string>
#include "tarch/Assertions.h"
namespace tarch { namespace logging {
class Log { public: explicit Log(const std::string&) {} };
}}
#define logWarning(fn, msg) do { if (0) { std::cerr << "warning " << fn << ": " << msg << std::endl; } } while (0)
#define logError(fn, msg) do { std::cerr << "error " << fn << ": " << msg << std::endl; } while (0)
#define logInfo(fn, msg) do { } while (0)
#define logDebug(fn, msg) do { } while (0)
