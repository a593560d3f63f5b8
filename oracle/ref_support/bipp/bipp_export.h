// Visibility macro for the oracle build of the reference sources.
#pragma once
#define BIPP_EXPORT __attribute__((visibility("default")))
#define BIPP_NO_EXPORT
