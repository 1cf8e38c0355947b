// Project-written stand-in for gtest/gtest_prod.h (gtest is not in the image).
// include/sketch.h only needs the FRIEND_TEST macro to exist.
#pragma once
#define FRIEND_TEST(test_case_name, test_name)
