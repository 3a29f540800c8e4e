// Stand-in version header: selects the RTC_FunctionRTC.hh include branch.
#pragma once
#define TRILINOS_MAJOR_MINOR_VERSION 130400
