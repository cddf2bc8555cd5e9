/* Shim used only to compile the reference engine on Linux: the reference includes
 * MFC's <afx.h> for CString, which it only uses as a file path (ofstream::open). */
#pragma once
#include <string>
typedef std::string CString;
