// logger_stub.cpp — stands in for the reference's src/logger.cpp when the
// reference's hot-path sources are compiled into oracle/_ref: that file needs
// boost/format.hpp (src/logger.cpp:16), which this image lacks.  Only the
// statics and Logger::open are defined, so WRITE_LOG lines (the Newton
// non-convergence notice) go to stdout only.
#include <string>
#include "logger.hpp"

namespace sph
{
std::string Logger::dir_name;
std::ofstream Logger::log_io;
bool Logger::open_flag = false;
void Logger::open(const std::string & output_dir) { dir_name = output_dir; }
void Logger::open(const char * output_dir) { dir_name = output_dir; }
}
