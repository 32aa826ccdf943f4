/* Stand-in for the Boost header included (but never used) by the reference's
 * parallel_filter_subsampling.cpp:4.  TEST INFRASTRUCTURE for oracle/_ref. */
#pragma once
