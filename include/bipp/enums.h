/* Processing unit, precision and log-level enumerations of the bipp C/C++ API.
 * The enumerators and their values are the reference's (include/bipp/enums.h:5-15),
 * kept identical so that callers of the reference compile against this library. */
#pragma once

enum BippProcessingUnit { BIPP_PU_AUTO, BIPP_PU_CPU, BIPP_PU_GPU };

enum BippPrecision { BIPP_PRECISION_SINGLE, BIPP_PRECISION_DOUBLE };

enum BippLogLevel {
  BIPP_LOG_LEVEL_OFF,
  BIPP_LOG_LEVEL_ERROR,
  BIPP_LOG_LEVEL_WARN,
  BIPP_LOG_LEVEL_INFO,
  BIPP_LOG_LEVEL_DEBUG,
};

#ifndef __cplusplus
typedef enum BippProcessingUnit BippProcessingUnit;
typedef enum BippLogLevel BippLogLevel;
typedef enum BippPrecision BippPrecision;
#endif
