/* Empty stand-in for the VMD molfile plugin header that the reference's
 * src/io_manager.h includes.  Nothing from it is used by the declarations the
 * reference's REMD driver (src/remd.cxx) needs; the plugin itself is not
 * vendored with the reference.  TEST INFRASTRUCTURE ONLY. */
#pragma once
