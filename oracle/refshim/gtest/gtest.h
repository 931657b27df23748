// Test infrastructure: the reference's encoder headers include gtest only to befriend their unit
// tests; this stand-in makes that declaration empty so that the encoders compile without gtest.
#pragma once
#define FRIEND_TEST(test_case, test_name)
