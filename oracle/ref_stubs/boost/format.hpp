/* Stand-in for a header the reference includes but this build does not need (no Boost here). */
#pragma once
