/* Test-infrastructure shim for building the reference CPU stepper on Linux.
 * The reference's logger.h includes the Windows-only <direct.h>; on Linux
 * nothing from it is needed, so this header is intentionally empty. */
#pragma once
