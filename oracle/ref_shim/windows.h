/* Empty stand-in: the reference includes <windows.h> on its WIN32 branch only for GetCoreCount. */
#pragma once
