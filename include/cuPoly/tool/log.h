// cuPoly's include/cuPoly/tool/log.h: a process-wide logger with a level.
// QUIET prints nothing; otherwise errors always print and the other messages
// print when their level is at or below the selected one (VERBOSE: all).
#ifndef LOG_H
#define LOG_H
#include <iostream>
#include <string>

enum log_mode { QUIET, INFO, WARNING, DEBUG, ERROR, VERBOSE };

class Logger {
 public:
  static Logger* getInstance() {
    static Logger instance;
    return &instance;
  }
  void set_mode(int m) { mode = m; }
  int get_mode() const { return mode; }
  void log_debug(const char* s) { print(s, DEBUG, "debug"); }
  void log_info(const char* s) { print(s, INFO, "info"); }
  void log_warning(const char* s) { print(s, WARNING, "warning"); }
  void log_error(const char* s) { print(s, ERROR, "error"); }

 private:
  Logger() = default;
  int mode = QUIET;
  void print(const char* s, int level, const char* name) {
    if (mode != QUIET && (mode == VERBOSE || level == ERROR || level <= mode)) std::cerr << "[cuPoly " << name << "] " << s << std::endl;
  }
};
#endif
