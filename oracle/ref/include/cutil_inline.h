/* Host-only stand-in (empty) for the NVIDIA SDK's cutil_inline.h. */
#pragma once
