"""B200-native Ros2 step and block-Thomas solve for VULCAN-style photochemistry."""
