// Error plumbing shared by the C-ABI translation units: every entry point
// body sits between EMG_API_BEGIN and EMG_API_END, which turn an emg::Error
// into its status code (and any other exception into EMG_ERR_USER) and keep
// the message for emg_last_error().
#pragma once

#include <exception>

#include "emg_internal.h"

namespace emg {
// argument and state checks of the entry points: fail with code unless cond
inline void need(bool cond, int code, const char *msg) {
  if (!cond) fail(code, "%s", msg);
}
}  // namespace emg

#define EMG_API_BEGIN try {
#define EMG_API_END                                  \
  }                                                  \
  catch (const emg::Error &e) {                      \
    emg::set_last_error(e.what());                   \
    return e.code;                                   \
  }                                                  \
  catch (const std::exception &e) {                  \
    emg::set_last_error(e.what());                   \
    return EMG_ERR_USER;                             \
  }                                                  \
  return EMG_OK;
