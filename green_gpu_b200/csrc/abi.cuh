// Exception barrier of the extern "C" entry points: every call returns a GG_* status and keeps
// the message (per context, or per thread for context-free calls) for gg_last_error().
#pragma once

#include "context.cuh"

namespace gg {

template <typename F>
int guarded(gg_context* c, F&& f) {
  if (!c) return GG_ERR_ARG;
  try {
    GG_CUDA(cudaSetDevice(c->device));
    f();
    c->err.clear();
    return GG_OK;
  } catch (const Error& e) {
    c->err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    c->err = e.what();
    return GG_ERR_INTERNAL;
  } catch (...) {
    c->err = "unknown error";
    return GG_ERR_INTERNAL;
  }
}

template <typename F>
int guarded_global(F&& f) {
  try {
    f();
    set_thread_error("");
    return GG_OK;
  } catch (const Error& e) {
    set_thread_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_thread_error(e.what());
    return GG_ERR_INTERNAL;
  } catch (...) {
    set_thread_error("unknown error");
    return GG_ERR_INTERNAL;
  }
}

}  // namespace gg
