/* Build configuration of the B200 implementation of the bipp C++ API. */
#pragma once
#define BIPP_CUDA
#define BIPP_VERSION "1.0.0-b200"
#ifndef BIPP_EXPORT
#define BIPP_EXPORT __attribute__((visibility("default")))
#endif
